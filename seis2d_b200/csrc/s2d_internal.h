// Internal layout and launch structures of libseis2d (not part of the ABI).
//
// Device layout of every per-cell field (state, materials):
//   element (x, z) of the padded grid lives at  base[(x + S2D_GX) * ld + (z + S2D_GZ)]
//   for x in [-S2D_GX, nnx + S2D_GX) and z in [-S2D_GZ, ld - S2D_GZ).
// Cells outside [0,nnx) x [0,nnz) are ghost cells: zero-filled once and never
// written, so that stencil reads near the grid edge need no branches.  The
// 1-D coefficient tables hold zeros at ghost indices, which makes every value
// the step computes at a ghost cell exactly zero.
#pragma once

#include <cstddef>
#include <cstdint>

#define S2D_GX 8            // ghost columns on each side
#define S2D_GZ 8            // ghost rows above z = 0
#define S2D_ZPT 4           // rows per lane (one float4)
#define S2D_STRIP_ROWS 128  // rows a warp reads (32 lanes x 4)
#define S2D_STRIP_OUT 120   // rows a one-step warp writes; strip k writes [120k, 120k+120), reads from 120k-4
#define S2D_TS_OUT 112      // rows a two-step warp writes; strip k writes [112k, 112k+112), reads from 112k-8

#if defined(__CUDACC__)
#define S2D_HD __host__ __device__
#else
#define S2D_HD
#endif

namespace s2d {

constexpr float kA0 = 1.125f;              // cpu_modelling_kernels.cpp:9
constexpr float kA1 = -1.0f / 24.0f;       // cpu_modelling_kernels.cpp:10 (float quotient)

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Strips a grid of nnz rows needs (one-step and two-step kernels), and the
// leading dimension that holds the rows either kind reads.
inline int num_strips(int nnz) { return (nnz + S2D_STRIP_OUT - 1) / S2D_STRIP_OUT; }
inline int num_strips_ts(int nnz) { return (nnz + S2D_TS_OUT - 1) / S2D_TS_OUT; }
inline int leading_dim(int nnz) {
    const int rows = S2D_STRIP_OUT * num_strips(nnz) > S2D_TS_OUT * num_strips_ts(nnz)
                         ? S2D_STRIP_OUT * num_strips(nnz)
                         : S2D_TS_OUT * num_strips_ts(nnz);
    return round_up(S2D_GZ + rows + 8, 32);
}

// One shot of a launch.  State pointers point at the allocation base
// (ghost origin); st[parity][field] with fields px, pz, vx, vz.  The eight
// state fields are one allocation, field k (= parity*4 + field) at
// st[0][0] + k*fstride, and kappa, bx, bz likewise (bx = kappa + fstride,
// bz = kappa + 2*fstride): the kernels address every field from one base.
struct ShotDev {
    float *st[2][4];
    const float *kappa, *bx, *bz;  // materials, same layout as the state
    const float4 *xcoef;           // [nnx + 2 GX]: damp2a, kx*damp2a1, damp2b, kx*damp2b1
    const float4 *zcoef;           // [ld]:         damp1a, kz*damp1a1, damp1b, kz*damp1b1
    int nnx, nnz, ld;
    int src_x, src_z;              // padded cell of the source
    const float *amp;              // [fd_nt] value added to px at the source after step kt
    const int *rec_ptr;            // [nnx + 1] receivers grouped by column (CSR)
    const int *rec_z;              // padded row of each receiver entry
    const int *rec_id;             // index of the entry's trace in seis
    float *seis;                   // [nrec][real_nt]; the adjoint reads its source here
    int real_nt;
    int fstride;                   // elements between consecutive fields (8 * fstride < 2^31)
    // gradient runs only
    float *prod;                   // [steps][4][field]: D-x vx, D-z vz, D+x p, D+z p of each step
    float *grad[2];                // accumulators dJ/dkappa, dJ/db (padded layout), one pair shared by the shots of a call
    float *srcadj;                 // [fd_nt] adjoint pressure at the source after each step
    float *scr;                    // 8th-order adjoint: Kx kappa mPX, Kz kappa mPZ (2 fields, ghosts 0)
    // element counts of the buffers above (device self-checks, S2D_DEVICE_CHECKS)
    size_t nfield;                 // every per-cell field
    size_t nprod;                  // prod
    size_t nseis;                  // seis (this shot's block)
    int nrec;
    // Rows [zfast_lo, zfast_hi) have the interior row constants: damp1a =
    // damp1b = 1, kz*damp1a1 = kz*damp1b1 = kz_in, operator pair (a0, a1).
    int zfast_lo, zfast_hi;
    float kz_in;
    // Columns [xfast_lo, xfast_hi) have the interior column constants:
    // damp2a = damp2b = 1, kx*damp2a1 = kx*damp2b1 = kx_in and both operator
    // pairs (a0, a1) (columns [2, nnx-3]).
    int xfast_lo, xfast_hi;
    float kx_in;
    int rec_zlo, rec_zhi;          // rows of the shot's receivers (rec_zlo > rec_zhi: none)
};

// Shots that share one grid shape; their tasks are interleaved so that the
// warps streaming the same tile of the same model for different shots run
// together and share the model's tiles through L2.
struct GroupDev {
    int task_begin;   // first flat task index of the group
    int nshots;       // shots in the group
    int shot0;        // index of the group's first shot in the shot table
    int nstrips;      // strips per shot
    int nsegs;        // x-segments per strip
    int seg_len;      // columns per x-segment
    int pad_[2];
};

// Arguments of one launch sequence.  They live in device memory and are
// written by a one-thread kernel in stream order before each sequence, so a
// captured graph of step launches serves every continuation and every shot.
struct StepArgs {
    const ShotDev *shots;
    const GroupDev *groups;
    int ngroups;
    int total_tasks;
    int dt_factor;
    int fd_nt;
    int kt_base;          // FD step of the launch with kt_off = 0
    int par0;             // state buffer holding step kt_base; launch kt_off reads par0 ^ (kt_off & 1)
    int stages;           // bulk-copy pipeline depth (shared-memory ring stages per warp)
    int *err;             // device error word (S2D_DEV_ERR_* bits), 0 when all waits completed
    int spin_limit;       // polls of an mbarrier before a wait counts as timed out
    int fault_iter;       // test knob: pipeline iteration whose copies are not issued (-1: none)
    int task_order;       // 0: shot fastest, 1: strip fastest (see task_of)
    int flags;            // S2D_STEP_* bits
    int prod_kt0;         // FD step stored in plane 0 of ShotDev::prod
    // TMA step kernel: tensor maps (CUtensorMap, 128 B each) of every shot's
    // 8 state planes in shot-table order, then of the 3 material planes of
    // every shot's model, in the same order; null for the other kernels
    const void *tmaps;
    int tmap_mat0;        // index of table slot 0's material map in tmaps
};

#define S2D_STEP_NO_RECORD 1  // forward: do not sample receivers; adjoint: do not inject the adjoint source
#define S2D_STEP_PRODUCTS 2   // forward also writes its four derivatives to ShotDev::prod

// Device error bits reported through StepArgs::err.
#define S2D_DEV_ERR_WAIT 1    // a pipeline wait gave up (bounded spin ran out)
#define S2D_DEV_ERR_DRAIN 2   // copies still in flight after the bounded drain

// Step kernel variants.
enum StepVariant { kVariantBulk = 0, kVariantLdg = 1, kVariantBulk128 = 2,
                   kVariantLdgProducts = 3 /* plain loads + S2D_STEP_PRODUCTS, gradient runs */,
                   kVariantLdg128 = 4 /* plain loads, compiled for 128 registers */,
                   kVariantTs2 = 5 /* two FD steps per launch (112-row strips) */,
                   kVariantTs1 = 6 /* one FD step in the two-step kernel's layout (odd remainders) */,
                   kVariantO8 = 7 /* 8th-order operator, plain loads (112-row strips), models with
                                     S2D_MODEL_ORDER8; 3 blocks per SM */,
                   kVariantO8r = 8 /* the same at 2 blocks per SM (no register cap below 224) */,
                   kVariantO8s = 9 /* the same with its windows in shared memory, 4 blocks per SM */,
                   kVariantO8Products = 10 /* kVariantO8 + S2D_STEP_PRODUCTS, gradient runs */,
                   kVariantTma = 11 /* CTA of kTmaWarps consumer warps fed by a TMA producer warp */,
                   kVariantAsync = 12 /* plain-load loop fed by per-lane cp.async into a per-warp ring */,
                   kVariantAsyncProducts = 13 /* kVariantAsync + S2D_STEP_PRODUCTS, gradient runs */,
                   kVariantLdgU4 = 14 /* kVariantLdg128 with its column loop unrolled by 4 */,
                   kVariantLdgPf = 15 /* plain loads, next column prefetched, 3 blocks per SM */,
                   kVariantLdgPf4 = 16 /* the same compiled for 4 blocks per SM */,
                   kVariantLdgPfU4 = 17 /* prefetch into two buffers in turn, unrolled by 4, 4 blocks per SM */,
                   kVariantLdgPfU3 = 18 /* the same compiled for 3 blocks per SM */,
                   kVariantLdgPfProducts = 19 /* kVariantLdgPf + S2D_STEP_PRODUCTS, gradient runs */,
                   kVariantPersist = 20 /* prefetching plain loads, many steps per cooperative launch */ };

// Per-warp ring of the async variant: kAsyncStages iterations of kAsyncSlots
// 128-row column slices (vx; px, pz, kappa, vz; bx, bz).
constexpr int kAsyncStages = 3;
constexpr int kAsyncSlots = 7;
constexpr int kAsyncWarpBytes = kAsyncStages * kAsyncSlots * S2D_STRIP_ROWS * 4;

// TMA step kernel: a CTA of kTmaWarps consumer warps (one 128-row strip of
// one shot each) and one producer warp that brings kTmaCols columns of the 7
// input slots of every consumer warp into a kTmaStages-deep shared-memory ring
// as 2-D tensor boxes of 128 rows x kTmaCols columns.
constexpr int kTmaWarps = 8;
constexpr int kTmaCols = 2;
constexpr int kTmaStages = 4;
constexpr int kTmaSlots = 7;  // vx at L; px, pz, kappa, vz at L-1; bx, bz at L-3
constexpr int kTmaBoxBytes = S2D_STRIP_ROWS * kTmaCols * 4;
constexpr int kTmaStageBytes = kTmaSlots * kTmaWarps * kTmaBoxBytes;
constexpr int kTmaThreads = (kTmaWarps + 1) * 32;
// ring, barriers and the slack that aligns the ring to 1 KB
constexpr size_t kTmaSmemBytes = (size_t)kTmaStages * kTmaStageBytes + 2 * kTmaStages * 8 + 1024;
constexpr int kTmaMapBytes = 128;  // sizeof(CUtensorMap)

// Tasks of a TMA launch: per group, blocks of kTmaWarps (shot, strip) pairs
// times x-segments.
S2D_HD inline int tma_blocks(int nshots, int nstrips) { return (nshots * nstrips + kTmaWarps - 1) / kTmaWarps; }

// FD steps one launch of a variant advances.
// (The persistent kernel runs any number of steps per launch; the autotuner's
// trial launches of it run 4.)
constexpr int kPersistTrialSteps = 4;
constexpr int steps_per_launch(int variant) {
    return variant == kVariantTs2 ? 2 : variant == kVariantPersist ? kPersistTrialSteps : 1;
}
// Variants whose strips are S2D_TS_OUT rows (and whose tasks stream 12 or 13 halo columns).
inline bool ts_layout(int variant) {
    return variant == kVariantTs2 || variant == kVariantTs1 || variant == kVariantO8 || variant == kVariantO8r ||
           variant == kVariantO8s || variant == kVariantO8Products;
}
inline bool order8_variant(int variant) {
    return variant == kVariantO8 || variant == kVariantO8r || variant == kVariantO8s;
}
inline bool tma_variant(int variant) { return variant == kVariantTma; }
inline bool async_variant(int variant) { return variant == kVariantAsync || variant == kVariantAsyncProducts; }
// Variants that use no dynamic shared memory.
inline bool plain_loads(int variant) {
    return variant == kVariantLdg || variant == kVariantLdgProducts || variant == kVariantLdg128 || variant == kVariantLdgU4 ||
           variant == kVariantLdgPf || variant == kVariantLdgPf4 || variant == kVariantLdgPfU4 ||
           variant == kVariantLdgPfU3 || variant == kVariantLdgPfProducts || variant == kVariantPersist ||
           variant == kVariantO8 || variant == kVariantO8r || variant == kVariantO8Products;
}

// Per-warp shared-memory delay lines of the two-step kernel (4 columns each):
// the first step's px, pz, vz and vx and the second step's p.
constexpr int kTsRing = 4;
constexpr int kTsFields = 5;
constexpr int kTsWarpBytes = kTsRing * kTsFields * S2D_STRIP_ROWS * 4;
// Per-warp shared-memory windows of the 8th-order ring kernel: vx and new p of
// 8 columns each, vz of 4 (one 128-row column = 32 float4).
constexpr int kO8sWarpBytes = (8 + 8 + 4) * S2D_STRIP_ROWS * 4;

// Shared memory of one pipeline stage: 7 slots of one 128-row column each
// (vx at L; px, pz, kappa, vz at L-1; bx, bz at L-3).
constexpr int kSlotBytes = S2D_STRIP_ROWS * 4;
constexpr int kSlots = 7;
constexpr int kStageBytes = kSlots * kSlotBytes;
inline size_t bulk_smem_bytes(int warps_per_block, int stages) {
    return (size_t)warps_per_block * stages * (kStageBytes + 8);
}

// Host-side launch helpers implemented in s2d_kernels.cu.
int launch_step(int variant, const StepArgs *args_dev, int kt_off, int grid, int block, size_t smem,
                void *stream);
int launch_set_args(const StepArgs &v, StepArgs *args_dev, void *stream);
// Persistent step kernel: `nsteps` FD steps from args->kt_base in one
// cooperative launch of `grid` blocks of 128 threads (all co-resident), with
// a grid barrier on the zeroed counter `bar` between steps.
int launch_persist(const StepArgs *args_dev, int nsteps, unsigned *bar, int grid, void *stream);
int persist_occupancy(int *blocks_per_sm);
// Adjoint FD step (step kt = args.kt_base - kt_off) and the gradient finalisation.
int launch_adjoint(const StepArgs *args_dev, int kt_off, int grid, int block, int minb, void *stream);
// Adjoint FD step of the 8th-order scheme: two cell-parallel passes over
// `nshots` shots of one nnx x nnz grid.
int launch_adjoint8(const StepArgs *args_dev, int kt_off, int nnx, int nnz, int nshots, void *stream);
// Adjoint FD step of the 8th-order scheme as one streaming pass (warp tasks on
// the 112-row strips of the batch's current layout), 4 warps per block.
int launch_adjoint8s(const StepArgs *args_dev, int kt_off, int grid, void *stream);
int adjoint8s_occupancy(int *blocks_per_sm);
int adjoint_kernel_occupancy(int block, int minb, int *blocks_per_sm);
// Add each shot's source term to its accumulator gk[s] (the entries may all
// be the one shared pair), sum the nacc accumulator pairs gk[0..nacc),
// gb[0..nacc) (dJ/dkappa, dJ/db), apply the kappa = vp^2 rho, b = 1/rho chain
// rule and fold the sponge onto the model.  kappa_fixed_rows: padded rows
// [0, kappa_fixed_rows) whose kappa is held at 0 (free surface), so their
// dJ/dkappa does not reach vp or rho.
int launch_gradient_finalize(float *const *gk, float *const *gb, int nshots, int nacc, const int *src_cells,
                             const double *src_vals, const float *vp, const float *rho, int nx, int nz, int nb,
                             int ld, int kappa_fixed_rows, float *tmp2, float *gvp_pad, float *grho_pad, float *grad_vp, float *grad_rho,
                             void *stream);
// Residual d - d_obs in place of d_obs... : res[i] = seis[i] - obs[i]; partial sums of res^2.
int launch_residual(const float *seis, const float *obs, float *res, size_t n, double *sumsq, void *stream);
int launch_prepare_model(const float *vp, const float *rho, int nx, int nz, int nb, int ld,
                         float *kappa, float *bue_scratch, float *bx, float *bz, void *stream);
int step_kernel_prepare(int variant, size_t smem);
int step_kernel_occupancy(int variant, int block, size_t smem, int *blocks_per_sm);
int step_kernel_attributes(int variant, int *regs, int *local_bytes);

}  // namespace s2d

// C ABI of libseis2d: contexts, models and the forward time loop.
//
// Replaces modelling_module() (src/src_cpu/modelling.h:106) for one device:
// the set-up of cpumodelling.cpp:168-292 is done once per model / run, and the
// shot loop of cpumodelling.cpp:326-380 becomes either one batched launch per
// FD step covering all shots (default) or the reference's shot-after-shot
// order (S2D_PLAIN).  The per-step launches are captured as a CUDA graph.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/seis2d.h"
#include "s2d_internal.h"
#include "s2d_setup.h"

using namespace s2d;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        reset();
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct Model {
    int nx = 0, nz = 0, nb = 0, nnx = 0, nnz = 0, ld = 0, nxa = 0;
    float dx = 0, dz = 0;
    bool free_surface = false;  // kappa held at 0 on padded rows 0..nb (S2D_MODEL_FREE_SURFACE)
    int fd_order = 4;            // 8 with S2D_MODEL_ORDER8
    size_t field_elems = 0;  // nxa * ld
    DevBuf vp, rho;          // raw [nx][nz] copies (source amplitude needs vp, rho at the source)
    DevBuf mat;              // kappa, bx, bz in one allocation, field_elems apart (padded layout)
    float *kappa() const { return mat.as<float>(); }
    float *bx() const { return mat.as<float>() + field_elems; }
    float *bz() const { return mat.as<float>() + 2 * field_elems; }
    std::vector<float> damp2a, damp2a1, damp2b, damp2b1, damp1a, damp1a1, damp1b, damp1b1;
    // Algorithmic DRAM bytes of one FD step of one shot: 44 B per cell, 36 B
    // where both pressure dampings are 1 (the cell carries p alone).
    double step_bytes() const {
        long cx = 0, cz = 0;
        for (int x = 0; x < nnx; ++x) cx += damp2a[x] == 1.0f;
        for (int z = 0; z < nnz; ++z) cz += damp1a[z] == 1.0f;
        const double merged = (double)cx * (double)cz, all = (double)nnx * (double)nnz;
        return 36.0 * merged + 44.0 * (all - merged);
    }
    // coefficient tables for one fd_dt, rebuilt when fd_dt changes
    float coef_dt = -1.0f;
    DevBuf xcoef, zcoef;
};

struct ShotHost {
    int model_id;
    int src_x, src_z;
    int nrec;
    size_t seis_off;  // element offset of the shot's [nrec][real_nt] block
};

struct Batch {
    int nshots = 0;
    bool plain = false;
    bool order8 = false;             // every shot's model has the 8th-order operator
    RunSteps steps{};
    int kt_next = 0;
    std::vector<ShotHost> shots;
    std::vector<ShotDev> shot_dev;   // host mirror
    std::vector<GroupDev> groups;    // batched mode
    std::vector<int> group_nnx;      // padded columns of each group's model
    std::vector<int> group_nnz;      // padded rows of each group's model
    int cur = 0;                     // state buffer (parity) holding step kt_next
    std::vector<long> layout;        // launch configuration the groups are laid out for
    std::vector<std::unique_ptr<DevBuf>> state;   // 8 per shot
    std::vector<std::unique_ptr<DevBuf>> aux;     // amp tables, receiver tables
    DevBuf shots_d, groups_d;
    DevBuf seis_int;                 // internal seismogram buffer (host output)
    float *seis_d = nullptr;         // where the kernels record
    size_t seis_elems = 0;
    long max_tasks = 0;              // largest task count of one launch sequence
    bool layout_tma = false;         // the groups are laid out in TMA tasks (kTmaWarps pairs each)
    std::vector<int> table;          // caller's shot index of each slot of the device shot table
    DevBuf tmaps_d;                  // TMA kernel: state maps per table slot, then material maps
};

// Device buffers of finished batches, kept for reuse by the next batch of
// the same sizes (state fields are the large allocations: a repeated run
// then needs no cudaMalloc).  Flushed when an allocation fails.
struct Pool {
    std::multimap<size_t, std::unique_ptr<DevBuf>> free;
    std::unique_ptr<DevBuf> take(size_t bytes, cudaError_t *err) {
        auto it = free.find(bytes);
        if (it != free.end()) {
            auto b = std::move(it->second);
            free.erase(it);
            *err = cudaSuccess;
            return b;
        }
        auto b = std::make_unique<DevBuf>();
        *err = b->alloc(bytes);
        if (*err == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            free.clear();
            *err = b->alloc(bytes);
        }
        return b;
    }
    void give(std::unique_ptr<DevBuf> b) {
        if (b && b->p) free.emplace(b->bytes, std::move(b));
    }
    size_t held() const {
        size_t n = 0;
        for (auto &kv : free) n += kv.first;
        return n;
    }
};

// Launch configuration of the step kernel.
struct LaunchCfg {
    int variant = kVariantLdgPf4;  // the fastest single configuration on the 64-shot 5000 x 5000 batch
    int block = 128;      // threads per block (whole warps)
    int stages = 3;       // bulk-copy ring depth per warp (bulk-copy variants)
    size_t smem = 0;
    int grid = 0;
    int order = -1;       // task order (StepArgs::task_order); -1: the context's option
};

struct Ctx {
    int device = 0;
    int sm_count = 0;
    // tuning options (s2d_set_option)
    // explicit launch configuration, used when autotuning is off
    int opt_variant = kVariantLdgPf4;
    int opt_variant8 = kVariantO8;  // 8th-order batches when autotuning is off
    int opt_block = 128;
    int opt_stages = 3;
    int opt_autotune = 1;     // time candidate configurations on a new batch shape
    int opt_seg_len = 0;      // 0 = automatic
    int opt_spin_limit = 1 << 20;
    int opt_fault_iter = -1;  // test knob, see s2d_set_option
    int opt_order = 1;        // task order (StepArgs::task_order)
    bool order_fixed = false; // task_order set by the caller: the autotuner keeps it
    int opt_grad_segment = 0; // gradient checkpoint interval, 0 = from free memory
    int opt_graph_chunk = 64; // FD steps per captured graph
    int opt_fast_rows = 1;    // 0: every strip takes the general row path
    int opt_adj_minb = 13;    // adjoint kernel build ("adjoint_blocks"): 3 blocks per SM, inputs by cp.async
    int opt_adj8_form = 0;    // 8th-order adjoint: 0 streaming pass, 1 two cell-parallel passes
    int opt_prod_variant = kVariantLdgPfProducts;  // s2d_gradient's product-writing forward (4th order)
    int last_segment = 0;     // interval the last gradient call used
    DevBuf dev_err;           // device error word of the step kernels
    DevBuf bar_d;             // grid-barrier counter of the persistent step kernel
    // Launch-argument block read by every step launch, and the graphs of step
    // launches captured against it (by step count and launch configuration);
    // kept for the context's lifetime, so later runs replay them.
    DevBuf args_d;
    std::map<std::vector<long>, cudaGraphExec_t> graphs;
    std::map<std::vector<long>, cudaGraphExec_t> adj_graphs;  // by (step count, grid)
    // autotuner results: batch shape -> (variant, block, stages)
    std::map<std::vector<long>, std::array<int, 4>> tuned;  // variant, block, stages, task order
    ~Ctx() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        for (auto &kv : adj_graphs) cudaGraphExecDestroy(kv.second);
    }
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // event pairs bracketing the phases of s2d_gradient (grown on demand)
    std::vector<cudaEvent_t> phase_ev;
    std::string err = "no error";
    std::map<int, std::unique_ptr<Model>> models;
    int next_model = 1;
    std::unique_ptr<Batch> batch;
    Pool pool;
    // Return the current batch's state buffers to the pool and drop it.
    void drop_batch() {
        if (!batch) return;
        for (auto &b : batch->state) pool.give(std::move(b));
        batch.reset();
    }
};

int fail(Ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(c, e_ == cudaErrorMemoryAllocation ? S2D_ERR_NOMEM : S2D_ERR_CUDA,    \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

// Columns per x-segment for a group.  Each task streams L + halo columns (6
// for one step per launch, 12 for two); warps loop over tasks, so a launch takes about
// ceil(tasks / resident warps) rounds of the longest task.  Pick the L with
// the fewest round-columns (longer segments on ties).
int choose_seg_len(int nnx, long tasks_per_seg, long resident_warps, int halo) {
    static const int cand[] = {1024, 768, 512, 384, 256, 192, 128, 96, 64, 48, 32, 24, 16, 12, 8, 6, 4};
    int best = 8;
    double best_cost = 1e300;
    for (int L : cand) {
        const int Lc = std::min(L, nnx);
        const long nsegs = (nnx + Lc - 1) / Lc;
        const long tasks = tasks_per_seg * nsegs;
        const long rounds = (tasks + resident_warps - 1) / std::max(1L, resident_warps);
        const double cost = (double)rounds * (Lc + halo);
        if (cost < best_cost * 0.999) {
            best_cost = cost;
            best = Lc;
        }
    }
    return best;
}

int build_coef(Ctx *c, Model &m, float fd_dt) {
    if (m.coef_dt == fd_dt && m.xcoef.p) return S2D_OK;
    const float inv_dx = 1.0f / m.dx, inv_dz = 1.0f / m.dz;
    const double dtdx = (double)(fd_dt * inv_dx), dtdz = (double)(fd_dt * inv_dz);
    std::vector<float4> xc(m.nxa), zc(m.ld);
    for (auto &v : xc) v = make_float4(0, 0, 0, 0);
    for (auto &v : zc) v = make_float4(0, 0, 0, 0);
    // kappaw2 = dtdx*kappa*damp2a1, buw2 = dtdx*bu2*damp2b1 (cpumodelling.cpp:270-281):
    // the per-column factors dtdx*damp?1 are folded here, kappa / b per cell in the kernel.
    for (int x = 0; x < m.nnx; ++x)
        xc[x + S2D_GX] = make_float4(m.damp2a[x], (float)(dtdx * m.damp2a1[x]), m.damp2b[x], (float)(dtdx * m.damp2b1[x]));
    for (int z = 0; z < m.nnz; ++z)
        zc[z + S2D_GZ] = make_float4(m.damp1a[z], (float)(dtdz * m.damp1a1[z]), m.damp1b[z], (float)(dtdz * m.damp1b1[z]));
    if (!m.xcoef.p) CK(m.xcoef.alloc(sizeof(float4) * m.nxa));
    if (!m.zcoef.p) CK(m.zcoef.alloc(sizeof(float4) * m.ld));
    CK(cudaMemcpyAsync(m.xcoef.p, xc.data(), sizeof(float4) * m.nxa, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(m.zcoef.p, zc.data(), sizeof(float4) * m.ld, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    m.coef_dt = fd_dt;
    return S2D_OK;
}

// Launch configuration for (variant, block, stages): shared memory and a grid
// of exactly the resident blocks (the kernels loop over tasks), capped by the
// work available.
int launch_config(Ctx *c, long max_tasks, LaunchCfg *out, int variant, int block, int stages) {
    LaunchCfg lc;
    lc.variant = variant;
    lc.block = std::max(32, std::min(128, block / 32 * 32));
    lc.stages = std::max(2, std::min(16, stages));
    const bool ldg = plain_loads(lc.variant);
    const bool ts = ts_layout(lc.variant);
    const bool tma = tma_variant(lc.variant);
    const bool asy = async_variant(lc.variant);
    if (ldg || ts || asy) {
        lc.block = 128;
        lc.stages = 0;
    }
    if (tma) {
        lc.block = kTmaThreads;
        lc.stages = 0;
    }
    lc.smem = ldg ? 0
              : tma ? kTmaSmemBytes
              : asy ? (size_t)(lc.block / 32) * kAsyncWarpBytes
              : ts ? (size_t)(lc.block / 32) * (lc.variant == kVariantO8s ? kO8sWarpBytes : kTsWarpBytes)
                   : bulk_smem_bytes(lc.block / 32, lc.stages);
    int e = step_kernel_prepare(lc.variant, lc.smem);
    if (e) return fail(c, S2D_ERR_ARG, "step kernel does not accept %zu B of shared memory: %s", lc.smem,
                       cudaGetErrorString((cudaError_t)e));
    int bps = 0;
    e = step_kernel_occupancy(lc.variant, lc.block, lc.smem, &bps);
    if (e || bps < 1)
        return fail(c, S2D_ERR_ARG, "launch configuration (variant %d, block %d, stages %d) cannot run", lc.variant,
                    lc.block, lc.stages);
    const long resident = (long)c->sm_count * bps;
    // warp tasks, or CTA tasks for the TMA kernel
    const long needed = tma ? max_tasks : (max_tasks * 32 + lc.block - 1) / lc.block;
    lc.grid = (int)std::max<long>(1, std::min<long>(resident, std::max<long>(needed, 1)));
    *out = lc;
    return S2D_OK;
}

// Key of a batch's shape for the autotuner: run mode and, per model group,
// padded grid and shot count.
std::vector<long> tune_key(const Ctx *c, const Batch &b) {
    std::vector<long> k = {b.plain ? 1L : 0L, (long)c->sm_count, b.order8 ? 8L : 4L};
    for (size_t g = 0; g < b.groups.size(); ++g) {
        k.push_back(b.group_nnx[g]);
        k.push_back(b.group_nnz[g]);
        k.push_back(b.groups[g].nshots);
    }
    return k;
}

// The configuration a run of batch `b` uses when it does not tune: the
// options when autotuning is off, else the tuned result for the batch's
// shape, else the built-in default.
int base_config(Ctx *c, const Batch &b, LaunchCfg *out, bool *tuned = nullptr) {
    if (tuned) *tuned = false;
    // 8th-order batches run the 8th-order kernel whatever the options say
    if (b.order8 && !c->opt_autotune) return launch_config(c, b.max_tasks, out, c->opt_variant8, 128, 0);
    if (!c->opt_autotune) return launch_config(c, b.max_tasks, out, c->opt_variant, c->opt_block, c->opt_stages);
    auto it = c->tuned.find(tune_key(c, b));
    if (it != c->tuned.end()) {
        if (tuned) *tuned = true;
        int e = launch_config(c, b.max_tasks, out, it->second[0], it->second[1], it->second[2]);
        out->order = c->order_fixed ? -1 : it->second[3];
        return e;
    }
    const LaunchCfg d;
    return launch_config(c, b.max_tasks, out, b.order8 ? kVariantO8 : d.variant, d.block, b.order8 ? 0 : d.stages);
}

// Segment lengths, segment counts and task ranges of the batch's groups for
// `resident_warps` warps looping over the tasks of a launch; uploaded when
// `key` differs from the layout in place.
// With `tma` a task is a CTA's: kTmaWarps (shot, strip) pairs of a group
// over one segment, and `resident_warps` counts resident CTAs.
int layout_groups_for(Ctx *c, Batch &b, long resident_warps, const std::vector<long> &key, bool ts = false,
                      bool tma = false) {
    if (b.layout == key) return S2D_OK;
    for (size_t gi = 0; gi < b.groups.size(); ++gi)
        b.groups[gi].nstrips = ts ? num_strips_ts(b.group_nnz[gi]) : num_strips(b.group_nnz[gi]);
    auto per_seg = [&](const GroupDev &g, int nshots) {
        return tma ? (long)tma_blocks(nshots, g.nstrips) : (long)nshots * g.nstrips;
    };
    long per_seg_total = 0;
    for (auto &g : b.groups) per_seg_total += per_seg(g, g.nshots);
    long max_tasks = 0;
    int task = 0;
    for (size_t gi = 0; gi < b.groups.size(); ++gi) {
        GroupDev &g = b.groups[gi];
        const int nnx = b.group_nnx[gi];
        // plain mode: every shot is a group of its own and runs alone
        const long tasks_per_seg = b.plain ? per_seg(g, 1) : per_seg_total;
        g.seg_len = c->opt_seg_len > 0 ? std::min(c->opt_seg_len, nnx)
                                       : choose_seg_len(nnx, tasks_per_seg, resident_warps, ts ? 12 : 6);
        g.nsegs = (nnx + g.seg_len - 1) / g.seg_len;
        if (b.plain) {
            g.task_begin = 0;
            max_tasks = std::max<long>(max_tasks, per_seg(g, 1) * g.nsegs);
        } else {
            g.task_begin = task;
            task += (int)(per_seg(g, g.nshots) * g.nsegs);
            max_tasks = task;
        }
    }
    if (!b.groups_d.p) CK(b.groups_d.alloc(sizeof(GroupDev) * b.groups.size()));
    CK(cudaMemcpyAsync(b.groups_d.p, b.groups.data(), sizeof(GroupDev) * b.groups.size(), cudaMemcpyHostToDevice,
                       c->stream));
    // the copy reads host memory that a later layout rewrites
    CK(cudaStreamSynchronize(c->stream));
    b.max_tasks = max_tasks;
    b.layout = key;
    b.layout_tma = tma;
    return S2D_OK;
}

// The layout for the resident warps of launch configuration `lc`.
int layout_groups(Ctx *c, Batch &b, const LaunchCfg &lc) {
    // the two-step kernel and its one-step companion share one layout
    const int v = lc.variant == kVariantTs1 ? kVariantTs2 : lc.variant;
    const std::vector<long> key = {v, lc.block, lc.stages, c->opt_seg_len};
    if (b.layout == key) return S2D_OK;
    // resident warps of the configuration (its grid when the work is smaller);
    // resident CTAs for the TMA kernel, whose tasks are CTA tasks
    LaunchCfg full;
    int e = launch_config(c, 1L << 40, &full, v, lc.block, lc.stages);
    if (e) return e;
    if (tma_variant(v)) return layout_groups_for(c, b, (long)full.grid, key, false, true);
    return layout_groups_for(c, b, (long)full.grid * (full.block / 32), key, ts_layout(v));
}

// Graph of `n` step launches (kt_off = 0..n-1) for one launch configuration,
// captured once per (n, configuration) and replayed; the launches read their
// step base from the device argument block written just before each replay.
int step_graph(Ctx *c, const LaunchCfg &lc, int n, cudaGraphExec_t *out) {
    StepArgs *args_d = c->args_d.as<StepArgs>();
    const std::vector<long> key = {n, lc.variant, lc.block, lc.stages, (long)lc.smem, lc.grid};
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < n; ++k) {
            int e = launch_step(lc.variant, args_d, k, lc.grid, lc.block, lc.smem, c->stream);
            if (e) {
                cudaStreamEndCapture(c->stream, &g);
                if (g) cudaGraphDestroy(g);
                return fail(c, S2D_ERR_CUDA, "step capture: %s", cudaGetErrorString((cudaError_t)e));
            }
        }
        CK(cudaStreamEndCapture(c->stream, &g));
        cudaGraphExec_t ge;
        cudaError_t ce = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        CK(ce);
        it = c->graphs.emplace(key, ge).first;
    }
    *out = it->second;
    return S2D_OK;
}

// Rows whose coefficients are the interior constants (see ShotDev::zfast_lo):
// damp1a = damp1b = 1, kz*damp1a1 = kz*damp1b1 = (float)kz, rows [2, nnz-3].
void fast_rows(const Model &m, float fd_dt, int *lo, int *hi, float *kz) {
    const double dtdz = (double)(fd_dt * (1.0f / m.dz));  // as build_coef forms it
    const float kzi = (float)(dtdz * 1.0f);
    auto ok = [&](int r) {
        return r >= 2 && r <= m.nnz - 3 && m.damp1a[r] == 1.0f && m.damp1b[r] == 1.0f &&
               (float)(dtdz * m.damp1a1[r]) == kzi && (float)(dtdz * m.damp1b1[r]) == kzi;
    };
    int a = 0;
    while (a < m.nnz && !ok(a)) ++a;
    int b = a;
    while (b < m.nnz && ok(b)) ++b;
    *lo = a;
    *hi = b;  // empty when a == b
    *kz = kzi;
}

// Columns whose coefficients are the interior constants (ShotDev::xfast_lo):
// damp2a = damp2b = 1, kx*damp2a1 = kx*damp2b1 = (float)kx and both operator
// pairs (a0, a1), columns [2, nnx-3].
void fast_cols(const Model &m, float fd_dt, int *lo, int *hi, float *kx) {
    const double dtdx = (double)(fd_dt * (1.0f / m.dx));  // as build_coef forms it
    const float kxi = (float)(dtdx * 1.0f);
    auto ok = [&](int x) {
        return x >= 2 && x <= m.nnx - 3 && m.damp2a[x] == 1.0f && m.damp2b[x] == 1.0f &&
               (float)(dtdx * m.damp2a1[x]) == kxi && (float)(dtdx * m.damp2b1[x]) == kxi;
    };
    int a = 0;
    while (a < m.nnx && !ok(a)) ++a;
    int b = a;
    while (b < m.nnx && ok(b)) ++b;
    *lo = a;
    *hi = b;  // empty when a == b
    *kx = kxi;
}

// One pass over `nsteps` FD steps starting at kt_begin, for the launch
// arguments `args` (a whole batch, or one shot of a plain run), as replays of
// a graph of `graph_chunk` launches.  The state at kt_begin is in buffer
// b.cur; each launch reads one buffer and writes the other, and b.cur follows.
// A two-step configuration finishes an odd count with one launch of its
// one-step companion (same strip layout).
// start_ev (direct launches only): recorded after the launch-argument update,
// just before the first step launch, so an interval timed from it holds the
// step kernels alone (the autotuner's trials).
int run_loop(Ctx *c, Batch &b, const LaunchCfg &lc, StepArgs args, int kt_begin, int nsteps, bool use_graph,
             int *launches, bool *graph_used, cudaEvent_t start_ev = nullptr) {
    if (nsteps <= 0) return S2D_OK;
    args.stages = lc.stages;
    args.err = c->dev_err.as<int>();
    args.spin_limit = c->opt_spin_limit;
    args.fault_iter = c->opt_fault_iter;
    args.task_order = lc.order >= 0 ? lc.order : c->opt_order;
    StepArgs *args_d = c->args_d.as<StepArgs>();
    if (lc.variant == kVariantPersist) {
        // chunks of graph_chunk steps, one cooperative launch each (not
        // captured: the launch itself covers the chunk)
        const int chunk = std::max(1, c->opt_graph_chunk);
        for (int done = 0; done < nsteps; done += chunk) {
            const int n = std::min(chunk, nsteps - done);
            args.kt_base = kt_begin + done;
            args.par0 = b.cur;
            int e = launch_set_args(args, args_d, c->stream);
            if (e) return fail(c, S2D_ERR_CUDA, "set_args launch: %s", cudaGetErrorString((cudaError_t)e));
            CK(cudaMemsetAsync(c->bar_d.p, 0, sizeof(unsigned), c->stream));
            e = launch_persist(args_d, n, c->bar_d.as<unsigned>(), lc.grid, c->stream);
            if (e) return fail(c, S2D_ERR_CUDA, "persistent step launch: %s", cudaGetErrorString((cudaError_t)e));
            *launches += 2;
            b.cur ^= n & 1;
        }
        return S2D_OK;
    }
    const int spl = steps_per_launch(lc.variant);
    const int nl = nsteps / spl, rem = nsteps - nl * spl;
    const int chunk = use_graph ? std::max(1, c->opt_graph_chunk) : std::max(nl, 1);
    for (int done = 0; done < nl; done += chunk) {
        const int n = std::min(chunk, nl - done);
        args.kt_base = kt_begin + done * spl;
        args.par0 = b.cur;
        int e = launch_set_args(args, args_d, c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "set_args launch: %s", cudaGetErrorString((cudaError_t)e));
        *launches += 1 + n;
        b.cur ^= n & 1;
        if (!use_graph) {
            if (start_ev) {
                CK(cudaEventRecord(start_ev, c->stream));
                start_ev = nullptr;
            }
            for (int k = 0; k < n; ++k) {
                e = launch_step(lc.variant, args_d, k, lc.grid, lc.block, lc.smem, c->stream);
                if (e) return fail(c, S2D_ERR_CUDA, "step launch: %s", cudaGetErrorString((cudaError_t)e));
            }
            continue;
        }
        cudaGraphExec_t ge;
        e = step_graph(c, lc, n, &ge);
        if (e) return e;
        CK(cudaGraphLaunch(ge, c->stream));
        *graph_used = true;
    }
    if (rem) {
        args.kt_base = kt_begin + nl * spl;
        args.par0 = b.cur;
        int e = launch_set_args(args, args_d, c->stream);
        if (!e) e = launch_step(kVariantTs1, args_d, 0, lc.grid, lc.block, lc.smem, c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "step launch: %s", cudaGetErrorString((cudaError_t)e));
        *launches += 2;
        b.cur ^= 1;
    }
    return S2D_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// Tensor map of `planes` per-cell fields of one grid, `fstride` elements
// apart from `base` (ghost origin): dims (row z + S2D_GZ, column x + S2D_GX,
// plane), boxes of 128 rows x kTmaCols columns.  The row extent stops at the
// grid's last row: boxes reaching past it read zeros without touching memory.
int encode_fields(Ctx *c, CUtensorMap *out, const float *base, int planes, const Model &m, size_t fstride) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return fail(c, S2D_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {(cuuint64_t)(m.nnz + S2D_GZ), (cuuint64_t)m.nxa, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)m.ld * sizeof(float), (cuuint64_t)fstride * sizeof(float)};
    const cuuint32_t box[3] = {S2D_STRIP_ROWS, kTmaCols, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box,
                           es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, S2D_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return S2D_OK;
}

// Tensor maps of a batch for the TMA step kernel, in device-table order: the
// 8 state planes of every shot, then the 3 material planes of every shot's
// model.
int build_tmaps(Ctx *c, Batch &b) {
    const int n = (int)b.table.size();
    static_assert(sizeof(CUtensorMap) == kTmaMapBytes, "tensor map size");
    std::vector<CUtensorMap> maps(2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        const int s = b.table[i];
        const Model &m = *c->models[b.shots[s].model_id];
        int e = encode_fields(c, &maps[i], b.shot_dev[s].st[0][0], 8, m, (size_t)b.shot_dev[s].fstride);
        if (!e) e = encode_fields(c, &maps[n + i], m.kappa(), 3, m, m.field_elems);
        if (e) return e;
    }
    CK(b.tmaps_d.alloc(sizeof(CUtensorMap) * maps.size()));
    CK(cudaMemcpy(b.tmaps_d.p, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice));
    return S2D_OK;
}

// Build the device tables of a new batch (kt_begin == 0).
int setup_batch(Ctx *c, const s2d_shot *shots, int nshots, const s2d_wave &wave, const double *wavelet,
                int nwavelet, float *seis_user, unsigned flags) {
    c->drop_batch();
    auto bp = std::make_unique<Batch>();
    Batch &b = *bp;
    b.nshots = nshots;
    b.plain = (flags & S2D_PLAIN) != 0;
    // every shot must reference an existing model; all share wave
    for (int s = 0; s < nshots; ++s) {
        auto it = c->models.find(shots[s].model_id);
        if (it == c->models.end()) return fail(c, S2D_ERR_ARG, "shot %d: unknown model id %d", s, shots[s].model_id);
        if (shots[s].nrec < 0 || (shots[s].nrec > 0 && !shots[s].rec))
            return fail(c, S2D_ERR_ARG, "shot %d: bad receiver list", s);
    }
    const Model &m0 = *c->models[shots[0].model_id];
    for (int s = 1; s < nshots; ++s)
        if (c->models[shots[s].model_id]->fd_order != m0.fd_order)
            return fail(c, S2D_ERR_ARG, "shot %d: the shots of one call must share the FD order (%d and %d)", s,
                        m0.fd_order, c->models[shots[s].model_id]->fd_order);
    b.order8 = m0.fd_order == 8;
    b.steps = derive_steps(wave, m0.dx, m0.dz);
    const RunSteps &rs = b.steps;
    if (rs.fd_nt < 1 || rs.real_nt < 1 || rs.dt_factor < 1)
        return fail(c, S2D_ERR_ARG, "bad time stepping: fd_nt=%d real_nt=%d dt_factor=%d", rs.fd_nt, rs.real_nt,
                    rs.dt_factor);
    // source wavelet: the reference Ricker (length nts, injected while kt <= nts,
    // the sample at kt == nts being 0) or the caller's samples
    std::vector<double> w;
    int inject_last;
    if (wavelet) {
        if (nwavelet < 0) return fail(c, S2D_ERR_ARG, "negative wavelet length");
        w.assign(wavelet, wavelet + nwavelet);
        inject_last = nwavelet - 1;
    } else {
        w = ricker(wave, rs.nts);
        inject_last = rs.nts;
    }
    size_t seis_total = 0;
    b.shots.resize(nshots);
    for (int s = 0; s < nshots; ++s) {
        Model &m = *c->models[shots[s].model_id];
        int e = build_coef(c, m, wave.fd_dt);
        if (e) return e;
        ShotHost &h = b.shots[s];
        h.model_id = shots[s].model_id;
        h.nrec = shots[s].nrec;
        cell_of(shots[s].src.x, shots[s].src.z, m.dx, m.dz, m.nb, h.src_x, h.src_z);
        if (h.src_x < 0 || h.src_x >= m.nnx || h.src_z < 0 || h.src_z >= m.nnz)
            return fail(c, S2D_ERR_GEOM, "shot %d: source (%g, %g) m is outside the grid", s, shots[s].src.x,
                        shots[s].src.z);
        h.seis_off = seis_total;
        seis_total += (size_t)h.nrec * rs.real_nt;
    }
    b.seis_elems = seis_total;
    if (flags & S2D_SEIS_DEVICE) {
        b.seis_d = seis_user;
    } else {
        CK(b.seis_int.alloc(std::max<size_t>(seis_total, 1) * sizeof(float)));
        b.seis_d = b.seis_int.as<float>();
    }
    if (seis_total) CK(cudaMemsetAsync(b.seis_d, 0, seis_total * sizeof(float), c->stream));

    b.shot_dev.resize(nshots);
    for (int s = 0; s < nshots; ++s) {
        Model &m = *c->models[shots[s].model_id];
        ShotHost &h = b.shots[s];
        ShotDev &d = b.shot_dev[s];
        std::memset(&d, 0, sizeof d);
        const size_t fb = m.field_elems * sizeof(float);
        // the 8 state fields of the shot in one allocation (ShotDev::fstride)
        {
            cudaError_t ae;
            b.state.push_back(c->pool.take(8 * fb, &ae));
            CK(ae);
            CK(cudaMemsetAsync(b.state.back()->p, 0, 8 * fb, c->stream));
            for (int par = 0; par < 2; ++par)
                for (int f = 0; f < 4; ++f)
                    d.st[par][f] = b.state.back()->as<float>() + (size_t)(par * 4 + f) * m.field_elems;
        }
        d.fstride = (int)m.field_elems;
        d.kappa = m.kappa();
        d.bx = m.bx();
        d.bz = m.bz();
        d.xcoef = m.xcoef.as<float4>();
        d.zcoef = m.zcoef.as<float4>();
        d.nnx = m.nnx;
        d.nnz = m.nnz;
        d.ld = m.ld;
        d.src_x = h.src_x;
        d.src_z = h.src_z;
        d.real_nt = rs.real_nt;
        d.seis = b.seis_d + h.seis_off;
        d.nfield = m.field_elems;
        d.nrec = h.nrec;
        d.nseis = (size_t)h.nrec * rs.real_nt;
        fast_rows(m, wave.fd_dt, &d.zfast_lo, &d.zfast_hi, &d.kz_in);
        fast_cols(m, wave.fd_dt, &d.xfast_lo, &d.xfast_hi, &d.kx_in);
        if (!c->opt_fast_rows) d.zfast_lo = d.zfast_hi = d.xfast_lo = d.xfast_hi = 0;
        // source amplitude per step: fd_dt * w[kt] * kappa[src] / (dx*dz)
        // (cpumodelling.cpp:136-140), kappa = vp^2 rho in double at the source
        const int mx = std::min(std::max(h.src_x - m.nb, 0), m.nx - 1);
        const int mz = std::min(std::max(h.src_z - m.nb, 0), m.nz - 1);
        float vr[2];
        CK(cudaMemcpy(&vr[0], m.vp.as<float>() + (size_t)mx * m.nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&vr[1], m.rho.as<float>() + (size_t)mx * m.nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
        // a source on the free surface or above it (kappa held at 0) injects nothing
        const double ksrc = m.free_surface && h.src_z <= m.nb ? 0.0 : ((double)vr[0] * (double)vr[0]) * (double)vr[1];
        const float dxdz = m.dx * m.dz;
        std::vector<float> amp(rs.fd_nt, 0.0f);
        for (int kt = 0; kt < rs.fd_nt && kt <= inject_last; ++kt) {
            const double wk = kt < (int)w.size() ? w[kt] : 0.0;
            amp[kt] = (float)(wave.fd_dt * wk * ksrc / dxdz);
        }
        // receivers grouped by column
        std::vector<int> rx(h.nrec), rz(h.nrec);
        for (int g = 0; g < h.nrec; ++g) {
            cell_of(shots[s].rec[g].x, shots[s].rec[g].z, m.dx, m.dz, m.nb, rx[g], rz[g]);
            if (rx[g] < 0 || rx[g] >= m.nnx || rz[g] < 0 || rz[g] >= m.nnz)
                return fail(c, S2D_ERR_GEOM, "shot %d receiver %d: (%g, %g) m is outside the grid", s, g,
                            shots[s].rec[g].x, shots[s].rec[g].z);
        }
        d.rec_zlo = m.nnz;
        d.rec_zhi = -1;
        for (int g = 0; g < h.nrec; ++g) {
            d.rec_zlo = std::min(d.rec_zlo, rz[g]);
            d.rec_zhi = std::max(d.rec_zhi, rz[g]);
        }
        std::vector<int> ptr(m.nnx + 1, 0), ez(h.nrec), eid(h.nrec);
        for (int g = 0; g < h.nrec; ++g) ptr[rx[g] + 1]++;
        for (int x = 0; x < m.nnx; ++x) ptr[x + 1] += ptr[x];
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int g = 0; g < h.nrec; ++g) {
            const int k = fill[rx[g]]++;
            ez[k] = rz[g];
            eid[k] = g;
        }
        b.aux.emplace_back(new DevBuf());
        DevBuf &ab = *b.aux.back();
        const size_t n_amp = (size_t)rs.fd_nt, n_ptr = (size_t)m.nnx + 1, n_rec = (size_t)std::max(h.nrec, 1);
        const size_t bytes = sizeof(float) * n_amp + sizeof(int) * (n_ptr + 2 * n_rec) + 64;
        CK(ab.alloc(bytes));
        char *base = ab.as<char>();
        float *amp_d = reinterpret_cast<float *>(base);
        int *ptr_d = reinterpret_cast<int *>(base + sizeof(float) * n_amp);
        int *ez_d = ptr_d + n_ptr;
        int *eid_d = ez_d + n_rec;
        CK(cudaMemcpy(amp_d, amp.data(), sizeof(float) * n_amp, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ptr_d, ptr.data(), sizeof(int) * n_ptr, cudaMemcpyHostToDevice));
        if (h.nrec) {
            CK(cudaMemcpy(ez_d, ez.data(), sizeof(int) * h.nrec, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(eid_d, eid.data(), sizeof(int) * h.nrec, cudaMemcpyHostToDevice));
        }
        d.amp = amp_d;
        d.rec_ptr = ptr_d;
        d.rec_z = ez_d;
        d.rec_id = eid_d;
    }
    CK(b.shots_d.alloc(sizeof(ShotDev) * nshots));
    CK(cudaMemcpy(b.shots_d.p, b.shot_dev.data(), sizeof(ShotDev) * nshots, cudaMemcpyHostToDevice));

    // groups: shots sharing a model, tasks interleaved over the group's shots.
    // In plain mode every shot is a group of its own and runs alone.
    std::vector<int> model_order;
    std::map<int, std::vector<int>> by_model;
    for (int s = 0; s < nshots; ++s) {
        if (!by_model.count(shots[s].model_id)) model_order.push_back(shots[s].model_id);
        by_model[shots[s].model_id].push_back(s);
    }
    if (b.plain) {
        for (int s = 0; s < nshots; ++s) b.table.push_back(s);
        for (int s = 0; s < nshots; ++s) {
            const Model &m = *c->models[shots[s].model_id];
            GroupDev g{};
            g.nshots = 1;
            g.shot0 = s;
            g.nstrips = num_strips(m.nnz);
            b.groups.push_back(g);
            b.group_nnx.push_back(m.nnx);
            b.group_nnz.push_back(m.nnz);
        }
    } else {
        // shots of one model must be contiguous in the shot table for shot0
        // indexing; keep the caller's order inside each model and reorder the
        // device table only (seis offsets stay the caller's).
        std::vector<ShotDev> reordered;
        for (int mid : model_order) {
            const Model &m = *c->models[mid];
            const std::vector<int> &ss = by_model[mid];
            GroupDev g{};
            g.nshots = (int)ss.size();
            g.shot0 = (int)reordered.size();
            g.nstrips = num_strips(m.nnz);
            b.groups.push_back(g);
            b.group_nnx.push_back(m.nnx);
            b.group_nnz.push_back(m.nnz);
            for (int s : ss) {
                reordered.push_back(b.shot_dev[s]);
                b.table.push_back(s);
            }
        }
        CK(cudaMemcpy(b.shots_d.p, reordered.data(), sizeof(ShotDev) * nshots, cudaMemcpyHostToDevice));
    }
    {
        int e = build_tmaps(c, b);
        if (e) return e;
    }
    // segment lengths for the configuration the run starts with
    {
        LaunchCfg lc;
        int e = base_config(c, b, &lc);
        if (!e) e = layout_groups(c, b, lc);
        if (e) return e;
    }
    CK(cudaStreamSynchronize(c->stream));
    c->batch = std::move(bp);
    return S2D_OK;
}

// Read and clear the step kernels' error word (after the stream is idle).
int check_device_error(Ctx *c) {
    int h = 0;
    CK(cudaMemcpy(&h, c->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        CK(cudaMemset(c->dev_err.p, 0, sizeof(int)));
        if (c->batch) c->batch->kt_next = -1;  // the wavefields are not valid any more
        return fail(c, S2D_ERR_TIMEOUT,
                    "a step-kernel pipeline wait ran out of its spin limit (device error bits 0x%x); "
                    "the affected steps were not computed",
                    h);
    }
    return S2D_OK;
}

}  // namespace

// Candidate launch configurations of the autotuner: (variant, block, stages,
// task order).  Task order 1 runs adjacent strips of one shot on the warps
// of a block; order 0 gives a block's warps the same strip and segment of
// consecutive shots, which then share the segment's kappa, bx, bz through
// the SM's L1 (the tasks of one launch are the same either way).
constexpr int kTuneCandidates[][4] = {
    {kVariantLdg128, 128, 0, 1}, {kVariantLdgPf4, 128, 0, 1}, {kVariantLdgPf, 128, 0, 1},
    {kVariantBulk128, 128, 3, 1}, {kVariantTs2, 128, 0, 1},    {kVariantTma, kTmaThreads, 0, 1},
    {kVariantAsync, 128, 0, 1},   {kVariantLdgPf4, 128, 0, 0}, {kVariantLdgPf, 128, 0, 0},
};
constexpr int kNumTuneCandidates = (int)(sizeof(kTuneCandidates) / sizeof(kTuneCandidates[0]));
// Candidates of 8th-order batches: the register-window kernel at 3 blocks per
// SM (168 registers) and at 2 (224 registers, no spills), and the
// shared-memory-window kernel at 4 (128 registers).
constexpr int kTuneCandidatesO8[][4] = {
    {kVariantO8, 128, 0, 1}, {kVariantO8r, 128, 0, 1}, {kVariantO8s, 128, 0, 1}, {kVariantO8, 128, 0, 0}};
constexpr int kNumTuneCandidatesO8 = (int)(sizeof(kTuneCandidatesO8) / sizeof(kTuneCandidatesO8[0]));
constexpr int kTuneWarm = 1, kTuneTimed = 3;  // launches per candidate
constexpr int kTuneRunoff = 4;                 // more timed launches of each of the two best
// FD steps the trials take (a two-step candidate advances two per launch).
constexpr int tune_steps(const int (*cand)[4], int n) {
    int steps = 0;
    for (int i = 0; i < n; ++i) steps += (kTuneWarm + kTuneTimed) * steps_per_launch(cand[i][0]);
    return steps;
}
// The most FD steps the trials and the runoff take (two two-step candidates
// in the runoff at most).
constexpr int kTuneSteps = tune_steps(kTuneCandidates, kNumTuneCandidates) + 2 * kTuneRunoff * 2;
constexpr int kTuneStepsO8 = tune_steps(kTuneCandidatesO8, kNumTuneCandidatesO8) + 2 * kTuneRunoff * 2;

// Sum of the task counts of a batched launch sequence.
int batch_tasks(const Batch &b) {
    int t = 0;
    for (auto &g : b.groups)
        t += (b.layout_tma ? tma_blocks(g.nshots, g.nstrips) : g.nshots * g.nstrips) * g.nsegs;
    return t;
}
// Tasks of shot s's own group in a plain run.
int plain_tasks(const Batch &b, int s) {
    const GroupDev &g = b.groups[s];
    return (b.layout_tma ? tma_blocks(1, g.nstrips) : g.nstrips) * g.nsegs;
}

// Autotuner: advance the batch by real FD steps from kt_begin (*steps_used
// of them, at most kTuneStepsMax): kTuneWarm + kTuneTimed launches under each
// candidate configuration, in rounds that visit every candidate once (every
// candidate computes the same bits: they share the update arithmetic and
// differ only in how columns reach registers, how many steps a pass makes and
// how tasks map to warps), with each timed launch between two events; then a
// runoff of kTuneRunoff more timed launches each, alternating, between the
// two candidates with the lowest median time per FD step, which decides
// between configurations whose medians lie within the trials' noise.  The
// winner is cached for the batch's shape and returned, its segment layout in
// place.
int autotune(Ctx *c, Batch &b, StepArgs a, int kt_begin, int *launches, LaunchCfg *best, int *steps_used) {
    const int (*const cands)[4] = b.order8 ? kTuneCandidatesO8 : kTuneCandidates;
    const int ncand = b.order8 ? kNumTuneCandidatesO8 : kNumTuneCandidates;
    const int nev = 2 * std::max(kTuneTimed * ncand, 2 * kTuneRunoff);
    std::vector<cudaEvent_t> ev(nev, nullptr);
    for (auto &e : ev) {
        cudaError_t ce = cudaEventCreate(&e);
        if (ce != cudaSuccess) {
            for (auto &x : ev)
                if (x) cudaEventDestroy(x);
            return fail(c, S2D_ERR_CUDA, "autotune events: %s", cudaGetErrorString(ce));
        }
    }
    struct Release {
        std::vector<cudaEvent_t> &ev;
        ~Release() {
            for (auto &x : ev) cudaEventDestroy(x);
        }
    } release{ev};
    std::vector<LaunchCfg> cfg(ncand), full(ncand);
    std::vector<bool> ok(ncand, false);
    for (int i = 0; i < ncand; ++i) {
        const int *k = cands[i];
        if (launch_config(c, 1L << 40, &full[i], k[0], k[1], k[2]) == S2D_OK) {
            ok[i] = true;
            full[i].order = c->order_fixed ? -1 : k[3];
        } else {
            if (i == 0) return S2D_ERR_ARG;
            // a configuration this device cannot run: its trial steps run
            // under the first candidate instead and are not counted
            full[i] = full[0];
        }
    }
    int kt = kt_begin;
    bool graph_used = false;
    // one launch of candidate i, timed between ev[e0] and ev[e0 + 1] when
    // e0 >= 0; the interval starts after the launch-argument update (a small
    // kernel of its own), so it holds the step launch alone
    auto trial = [&](int i, int e0) -> int {
        LaunchCfg lc = full[i];
        int e = layout_groups(c, b, lc);
        if (!e) e = launch_config(c, b.max_tasks, &lc, lc.variant, lc.block, lc.stages);
        if (e) return e;
        lc.order = full[i].order;
        cfg[i] = lc;
        a.total_tasks = batch_tasks(b);
        const int spl = steps_per_launch(lc.variant);
        e = run_loop(c, b, lc, a, kt, spl, false, launches, &graph_used, e0 >= 0 ? ev[e0] : nullptr);
        if (e) return e;
        if (e0 >= 0) CK(cudaEventRecord(ev[e0 + 1], c->stream));
        kt += spl;
        return S2D_OK;
    };
    // Rounds: one untimed, then kTuneTimed timed, each visiting every
    // candidate once, so clock ramps and drift reach all candidates alike.
    for (int r = 0; r < kTuneWarm + kTuneTimed; ++r) {
        const int t = r - kTuneWarm;
        for (int i = 0; i < ncand; ++i) {
            int e = trial(i, t >= 0 ? 2 * (i * kTuneTimed + t) : -1);
            if (e) return e;
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    int pick = 0, second = -1;
    float pick_ms = 0, second_ms = 0;
    for (int i = 0; i < ncand; ++i) {
        float t[kTuneTimed];
        for (int s = 0; s < kTuneTimed; ++s)
            CK(cudaEventElapsedTime(&t[s], ev[2 * (i * kTuneTimed + s)], ev[2 * (i * kTuneTimed + s) + 1]));
        std::sort(t, t + kTuneTimed);
        const float med = t[kTuneTimed / 2] / (float)steps_per_launch(cfg[i].variant);  // per FD step
        if (!ok[i]) continue;
        if (i == 0 || med < pick_ms) {
            second = i == 0 ? -1 : pick;
            second_ms = pick_ms;
            pick = i;
            pick_ms = med;
        } else if (second < 0 || med < second_ms) {
            second = i;
            second_ms = med;
        }
    }
    // runoff between the two best: kTuneRunoff timed launches each, alternating
    if (second >= 0) {
        const int two[2] = {pick, second};
        for (int r = 0; r < kTuneRunoff; ++r)
            for (int q = 0; q < 2; ++q) {
                int e = trial(two[q], 2 * (r * 2 + q));
                if (e) return e;
            }
        CK(cudaStreamSynchronize(c->stream));
        float tot[2] = {0.0f, 0.0f};
        for (int r = 0; r < kTuneRunoff; ++r)
            for (int q = 0; q < 2; ++q) {
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, ev[2 * (r * 2 + q)], ev[2 * (r * 2 + q) + 1]));
                tot[q] += ms / (float)steps_per_launch(cfg[two[q]].variant);
            }
        if (tot[1] < tot[0]) pick = second;
    }
    *steps_used = kt - kt_begin;
    const int *k = cands[pick];
    c->tuned[tune_key(c, b)] = {k[0], k[1], k[2], full[pick].order};
    int e = layout_groups(c, b, cfg[pick]);
    if (!e) e = launch_config(c, b.max_tasks, best, k[0], k[1], k[2]);
    best->order = full[pick].order;
    return e;
}

// ---------------------------------------------------------------------------

extern "C" {

int s2d_abi_version(void) { return S2D_ABI_VERSION; }

int s2d_set_option(void *ctx, const char *key, long value) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c || !key) return S2D_ERR_ARG;
    const std::string k(key);
    // an explicit launch configuration turns the autotuner off
    if (k == "variant") {
        if (order8_variant((int)value)) {
            // the 8th-order kernels serve 8th-order batches only
            c->opt_variant8 = (int)value;
            c->opt_autotune = 0;
            return S2D_OK;
        }
        if (value != kVariantBulk && value != kVariantLdg && value != kVariantBulk128 && value != kVariantLdg128 &&
            value != kVariantTs2 && value != kVariantTma && value != kVariantAsync && value != kVariantLdgU4 &&
            value != kVariantLdgPf && value != kVariantLdgPf4 && value != kVariantLdgPfU4 &&
            value != kVariantLdgPfU3 && value != kVariantPersist)
            return fail(c, S2D_ERR_ARG, "unknown step kernel variant %ld", value);
        c->opt_variant = (int)value;
        c->opt_autotune = 0;
    } else if (k == "block") {
        if (value < 32 || value > 128 || value % 32)
            return fail(c, S2D_ERR_ARG, "block must be 1 to 4 whole warps (the step kernels are built for <= 128 threads)");
        c->opt_block = (int)value;
        c->opt_autotune = 0;
    } else if (k == "stages") {
        if (value < 2 || value > 16) return fail(c, S2D_ERR_ARG, "stages must be in [2, 16]");
        c->opt_stages = (int)value;
        c->opt_autotune = 0;
    } else if (k == "seg_len") {
        if (value < 0) return fail(c, S2D_ERR_ARG, "seg_len must be >= 0");
        c->opt_seg_len = (int)value;
    } else if (k == "autotune") {
        if (value != 0 && value != 1) return fail(c, S2D_ERR_ARG, "autotune must be 0 or 1");
        c->opt_autotune = (int)value;
    } else if (k == "spin_limit") {
        if (value < 1) return fail(c, S2D_ERR_ARG, "spin_limit must be >= 1");
        c->opt_spin_limit = (int)std::min<long>(value, 1L << 30);
    } else if (k == "adjoint8_form") {
        if (value != 0 && value != 1) return fail(c, S2D_ERR_ARG, "adjoint8_form must be 0 or 1");
        c->opt_adj8_form = (int)value;
    } else if (k == "products_variant") {
        if (value != kVariantLdgProducts && value != kVariantLdgPfProducts)
            return fail(c, S2D_ERR_ARG, "products_variant must be %d or %d", kVariantLdgProducts, kVariantLdgPfProducts);
        c->opt_prod_variant = (int)value;
    } else if (k == "adjoint_blocks") {
        if ((value < 2 || value > 4) && (value < 12 || value > 15))
            return fail(c, S2D_ERR_ARG,
                        "adjoint_blocks must be 2, 3, 4, 12 (2 with the next column prefetched), 13, 14 or 15 (3, 2 "
                        "or 3 blocks with asynchronous copies 1, 2 or 2 columns ahead)");
        c->opt_adj_minb = (int)value;
    } else if (k == "fast_rows") {
        c->opt_fast_rows = value ? 1 : 0;
    } else if (k == "graph_chunk") {
        if (value < 1 || value > 100000) return fail(c, S2D_ERR_ARG, "graph_chunk must be in [1, 100000]");
        c->opt_graph_chunk = (int)value;
    } else if (k == "grad_segment") {
        if (value < 0) return fail(c, S2D_ERR_ARG, "grad_segment must be >= 0");
        c->opt_grad_segment = (int)value;
    } else if (k == "task_order") {
        if (value != 0 && value != 1) return fail(c, S2D_ERR_ARG, "task_order must be 0 or 1");
        c->opt_order = (int)value;
        c->order_fixed = true;
    } else if (k == "inject_wait_fault") {
        c->opt_fault_iter = value < 0 ? -1 : (int)value;
    } else {
        return fail(c, S2D_ERR_ARG, "unknown option '%s'", key);
    }
    return S2D_OK;
}

int s2d_derive_steps(const s2d_wave *wave, s2d_steps *out) {
    if (!wave || !out) return S2D_ERR_ARG;
    if (!(wave->fd_dt > 0) || !(wave->real_dt > 0) || !(wave->rec_len > 0) || !(wave->dom_freq > 0)) return S2D_ERR_ARG;
    RunSteps r = derive_steps(*wave, 1.0f, 1.0f);
    out->fd_nt = r.fd_nt;
    out->real_nt = r.real_nt;
    out->dt_factor = r.dt_factor;
    out->nts = r.nts;
    return S2D_OK;
}

int s2d_create(void **ctx, int device) {
    if (!ctx) return S2D_ERR_ARG;
    *ctx = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return S2D_ERR_NODEV;
    }
    if (device < 0 || device >= n) return S2D_ERR_ARG;
    auto c = new Ctx();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = c->dev_err.alloc(sizeof(int));
    if (e == cudaSuccess) e = c->bar_d.alloc(sizeof(unsigned));
    if (e == cudaSuccess) e = c->args_d.alloc(sizeof(StepArgs));
    if (e == cudaSuccess) e = cudaMemset(c->dev_err.p, 0, sizeof(int));
    if (e != cudaSuccess) {
        delete c;
        cudaGetLastError();
        return S2D_ERR_CUDA;
    }
    *ctx = c;
    return S2D_OK;
}

void s2d_destroy(void *ctx) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->batch.reset();
    c->pool.free.clear();
    c->models.clear();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (cudaEvent_t e : c->phase_ev) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *s2d_last_error(const void *ctx) {
    const Ctx *c = static_cast<const Ctx *>(ctx);
    return c ? c->err.c_str() : "null context";
}

int s2d_model_create(void *ctx, int nx, int nz, float dx, float dz, int nb, const float *vp, const float *rho,
                     unsigned flags, int *model_id) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c) return S2D_ERR_ARG;
    if (!vp || !rho || !model_id) return fail(c, S2D_ERR_ARG, "null model pointer");
    if (nx < 1 || nz < 1 || nb < 2 || !(dx > 0) || !(dz > 0))
        return fail(c, S2D_ERR_ARG, "bad model shape nx=%d nz=%d nb=%d dx=%g dz=%g", nx, nz, nb, dx, dz);
    CK(cudaSetDevice(c->device));
    auto m = std::make_unique<Model>();
    m->nx = nx; m->nz = nz; m->nb = nb; m->dx = dx; m->dz = dz;
    m->fd_order = (flags & S2D_MODEL_ORDER8) ? 8 : 4;
    m->nnx = nx + 2 * nb;
    m->nnz = nz + 2 * nb;
    m->ld = leading_dim(m->nnz);
    m->nxa = m->nnx + 2 * S2D_GX;
    m->field_elems = (size_t)m->nxa * m->ld;
    // kernels address the 8 state fields of a shot with 32-bit offsets
    if (8 * m->field_elems >= (size_t)1 << 31)
        return fail(c, S2D_ERR_ARG, "padded grid %d x %d is too large (8 fields of %zu cells exceed 2^31)", m->nnx,
                    m->nnz, m->field_elems);
    // the per-cell set-up and gradient kernels put one padded column per grid row
    if (m->nnx > 65535)
        return fail(c, S2D_ERR_ARG, "padded grid has %d columns; at most 65535 are supported", m->nnx);
    const size_t raw = (size_t)nx * nz * sizeof(float);
    CK(m->vp.alloc(raw));
    CK(m->rho.alloc(raw));
    const cudaMemcpyKind kind = (flags & S2D_MODEL_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(cudaMemcpyAsync(m->vp.p, vp, raw, kind, c->stream));
    CK(cudaMemcpyAsync(m->rho.p, rho, raw, kind, c->stream));
    const size_t fb = m->field_elems * sizeof(float);
    CK(m->mat.alloc(3 * fb));
    DevBuf bue;
    CK(bue.alloc(fb));
    CK(cudaMemsetAsync(m->mat.p, 0, 3 * fb, c->stream));
    CK(cudaMemsetAsync(bue.p, 0, fb, c->stream));
    int e = launch_prepare_model(m->vp.as<float>(), m->rho.as<float>(), nx, nz, nb, m->ld, m->kappa(), bue.as<float>(),
                                 m->bx(), m->bz(), c->stream);
    if (e) return fail(c, S2D_ERR_CUDA, "prepare_model: %s", cudaGetErrorString((cudaError_t)e));
    if (flags & S2D_MODEL_FREE_SURFACE) {
        // vacuum form of a pressure-release surface: kappa = 0 on padded rows
        // 0..nb of every column, so p stays 0 on the surface row and above it
        m->free_surface = true;
        CK(cudaMemset2DAsync(m->kappa() + (size_t)S2D_GX * m->ld + S2D_GZ, sizeof(float) * m->ld, 0,
                             sizeof(float) * (nb + 1), m->nnx, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    sponge_a(nb, nx, m->damp2a, m->damp2a1);
    sponge_b(nb, nx, m->damp2b, m->damp2b1);
    sponge_a(nb, nz, m->damp1a, m->damp1a1);
    sponge_b(nb, nz, m->damp1b, m->damp1b1);
    const int id = c->next_model++;
    c->models[id] = std::move(m);
    *model_id = id;
    return S2D_OK;
}

int s2d_model_destroy(void *ctx, int model_id) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c) return S2D_ERR_ARG;
    auto it = c->models.find(model_id);
    if (it == c->models.end()) return fail(c, S2D_ERR_ARG, "unknown model id %d", model_id);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->drop_batch();  // a batch may reference the model
    c->models.erase(it);
    return S2D_OK;
}

int s2d_forward(void *ctx, const s2d_shot *shots, int nshots, const s2d_wave *wave, const double *wavelet,
                int nwavelet, int kt_begin, int kt_count, float *seis_out, unsigned flags, s2d_stats *stats) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c) return S2D_ERR_ARG;
    if (!shots || nshots < 1 || !wave) return fail(c, S2D_ERR_ARG, "no shots or no wave description");
    if (!seis_out) return fail(c, S2D_ERR_ARG, "null seismogram buffer");
    if (!(wave->fd_dt > 0) || !(wave->real_dt > 0) || !(wave->rec_len > 0) || !(wave->dom_freq > 0))
        return fail(c, S2D_ERR_ARG, "wave parameters must be positive");
    if (kt_begin < 0) return fail(c, S2D_ERR_ARG, "negative kt_begin");
    CK(cudaSetDevice(c->device));
    if (kt_begin == 0) {
        int e = setup_batch(c, shots, nshots, *wave, wavelet, nwavelet, seis_out, flags);
        if (e) {
            c->drop_batch();
            return e;
        }
    } else {
        if (!c->batch || c->batch->nshots != nshots || c->batch->kt_next != kt_begin ||
            c->batch->plain != ((flags & S2D_PLAIN) != 0))
            return fail(c, S2D_ERR_STATE, "continuation at kt=%d does not follow the previous call", kt_begin);
        if (flags & S2D_SEIS_DEVICE) {
            if (c->batch->seis_d != seis_out)
                return fail(c, S2D_ERR_STATE, "continuation must record into the same device buffer");
        }
    }
    Batch &b = *c->batch;
    const RunSteps &rs = b.steps;
    const int kt_end = (kt_count <= 0) ? rs.fd_nt : std::min(rs.fd_nt, kt_begin + kt_count);
    const int nsteps = kt_end - kt_begin;
    if (nsteps < 0) return fail(c, S2D_ERR_ARG, "kt_begin %d beyond fd_nt %d", kt_begin, rs.fd_nt);
    const bool use_graph = !(flags & S2D_NO_GRAPH);
    int launches = 0;
    bool graph_used = false;
    bool tuned = false;
    LaunchCfg lc;
    {
        int e = base_config(c, b, &lc, &tuned);
        const int order = lc.order;
        if (!e) e = layout_groups(c, b, lc);
        if (!e) e = launch_config(c, b.max_tasks, &lc, lc.variant, lc.block, lc.stages);
        if (e) return e;
        lc.order = order;
    }
    CK(cudaEventRecord(c->ev0, c->stream));
    StepArgs a{};
    a.shots = b.shots_d.as<ShotDev>();
    a.dt_factor = rs.dt_factor;
    a.fd_nt = rs.fd_nt;
    a.tmaps = b.tmaps_d.p;
    a.tmap_mat0 = b.nshots;
    int kt_run = kt_begin;  // first step left after tuning
    int tuned_now = 0;
    // Batched runs of a shape with no tuned configuration yet tune on their
    // first steps when the call has room for the trials and a run after them.
    const int tune_len = b.order8 ? kTuneStepsO8 : kTuneSteps;
    if (c->opt_autotune && !tuned && !b.plain && nsteps >= 2 * tune_len) {
        a.groups = b.groups_d.as<GroupDev>();
        a.ngroups = (int)b.groups.size();
        int used = 0;
        int e = autotune(c, b, a, kt_begin, &launches, &lc, &used);
        if (e) return e;
        kt_run += used;
        tuned_now = 1;
    }
    if (b.plain) {
        // every shot advances from the same buffer through the same launches
        const int cur0 = b.cur;
        for (int s = 0; s < nshots; ++s) {
            a.groups = b.groups_d.as<GroupDev>() + s;
            a.ngroups = 1;
            a.total_tasks = plain_tasks(b, s);
            b.cur = cur0;
            int e = run_loop(c, b, lc, a, kt_begin, nsteps, use_graph, &launches, &graph_used);
            if (e) return e;
        }
    } else {
        a.groups = b.groups_d.as<GroupDev>();
        a.ngroups = (int)b.groups.size();
        a.total_tasks = batch_tasks(b);
        int e = run_loop(c, b, lc, a, kt_run, kt_end - kt_run, use_graph, &launches, &graph_used);
        if (e) return e;
    }
    CK(cudaEventRecord(c->ev1, c->stream));
    b.kt_next = kt_end;
    // seismogram samples recorded in [kt_begin, kt_end), widened to the whole
    // trace at the run's start and end so unrecorded samples read as zero
    if (!(flags & S2D_SEIS_DEVICE) && b.seis_elems) {
        int t0 = kt_begin == 0 ? 0 : (kt_begin + 1 + rs.dt_factor - 1) / rs.dt_factor - 1;
        int t1 = kt_end >= rs.fd_nt ? rs.real_nt : kt_end / rs.dt_factor;
        t0 = std::max(0, std::min(t0, rs.real_nt));
        t1 = std::max(t0, std::min(t1, rs.real_nt));
        if (t1 > t0) {
            const size_t rows = b.seis_elems / rs.real_nt;
            if (t1 - t0 == rs.real_nt) {
                // whole traces: one contiguous copy (a copy of one row per
                // trace would take the copy engine row by row)
                CK(cudaMemcpyAsync(seis_out, b.seis_d, sizeof(float) * b.seis_elems, cudaMemcpyDeviceToHost,
                                   c->stream));
            } else {
                CK(cudaMemcpy2DAsync(seis_out + t0, sizeof(float) * rs.real_nt, b.seis_d + t0,
                                     sizeof(float) * rs.real_nt, sizeof(float) * (t1 - t0), rows,
                                     cudaMemcpyDeviceToHost, c->stream));
            }
        }
        CK(cudaStreamSynchronize(c->stream));
    } else if (flags & S2D_SYNC) {
        CK(cudaStreamSynchronize(c->stream));
    }
    if (!(flags & S2D_SEIS_DEVICE) || (flags & S2D_SYNC)) {
        int e = check_device_error(c);
        if (e) return e;
    }
    if (stats) {
        CK(cudaEventSynchronize(c->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        double cells = 0, bytes = 0;
        for (int s = 0; s < nshots; ++s) {
            const Model &m = *c->models[b.shots[s].model_id];
            cells += (double)m.nnx * m.nnz;
            bytes += m.step_bytes();
        }
        stats->loop_ms = ms;
        stats->cell_updates = cells * nsteps;
        // one pass over the state per launch (two steps per pass for the
        // two-step kernel; the autotuner's trial steps are counted as one-step)
        const int passes = steps_per_launch(lc.variant) == 2 ? (kt_end - kt_run + 1) / 2 + (kt_run - kt_begin)
                                                             : nsteps;
        stats->alg_bytes = bytes * passes;
        stats->gcells_per_s = ms > 0 ? stats->cell_updates / (ms * 1e6) : 0.0;
        stats->kernel_launches = launches;
        stats->graph_used = graph_used ? 1 : 0;
        stats->grad_segment = 0;
        stats->sweep_ms = stats->recompute_ms = stats->adjoint_ms = 0;
        stats->task_order = lc.order >= 0 ? lc.order : c->opt_order;
        stats->variant = lc.variant;
        stats->block = lc.block;
        stats->stages = lc.stages;
        stats->seg_len = b.groups.empty() ? 0 : b.groups[0].seg_len;
        stats->autotuned = tuned_now;
    }
    return S2D_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Gradient (adjoint state with checkpointed forward recompute)

namespace {

struct GradRun {
    std::vector<std::unique_ptr<DevBuf>> bufs;
    // phase boundaries: (phase, index into Ctx::phase_ev); the time from one
    // mark to the next counts for the first mark's phase
    std::vector<std::pair<int, int>> marks;
};
enum { kPhaseOther = 0, kPhaseSweep = 1, kPhaseRecompute = 2, kPhaseAdjoint = 3 };

int phase_mark(Ctx *c, GradRun &g, int phase) {
    const int i = (int)g.marks.size();
    if (i == (int)c->phase_ev.size()) {
        cudaEvent_t e;
        CK(cudaEventCreate(&e));
        c->phase_ev.push_back(e);
    }
    CK(cudaEventRecord(c->phase_ev[i], c->stream));
    g.marks.emplace_back(phase, i);
    return S2D_OK;
}

int grad_alloc(Ctx *c, GradRun &g, size_t bytes, void **out) {
    cudaError_t e;
    g.bufs.push_back(c->pool.take(bytes, &e));
    CK(e);
    *out = g.bufs.back()->p;
    return S2D_OK;
}

// Adjoint launches for steps kt_top, kt_top-1, ..., kt_top-n+1, as replays of
// a graph of `graph_chunk` launches.
// The 8th-order adjoint over steps kt_top, kt_top-1, ..., kt_top-n+1: two
// cell-parallel launches per step, direct (no graph).
int run_adjoint8(Ctx *c, StepArgs args, int kt_top, int n, int nnx, int nnz, int nshots, int *launches) {
    if (n <= 0) return S2D_OK;
    StepArgs *args_d = c->args_d.as<StepArgs>();
    args.kt_base = kt_top;
    int e = launch_set_args(args, args_d, c->stream);
    if (e) return fail(c, S2D_ERR_CUDA, "set_args launch: %s", cudaGetErrorString((cudaError_t)e));
    if (c->opt_adj8_form == 0) {
        // one streaming pass per step over the warp tasks of the current
        // (112-row) layout, the grid exactly its resident blocks
        int bps = 0;
        if (adjoint8s_occupancy(&bps) || bps < 1) bps = 1;
        const int grid = (int)std::max<long>(
            1, std::min<long>((long)c->sm_count * bps, ((long)args.total_tasks * 32 + 127) / 128));
        *launches += 1 + n;
        for (int k = 0; k < n; ++k) {
            e = launch_adjoint8s(args_d, k, grid, c->stream);
            if (e) return fail(c, S2D_ERR_CUDA, "adjoint launch: %s", cudaGetErrorString((cudaError_t)e));
        }
        return S2D_OK;
    }
    *launches += 1 + 2 * n;
    for (int k = 0; k < n; ++k) {
        e = launch_adjoint8(args_d, k, nnx, nnz, nshots, c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "adjoint launch: %s", cudaGetErrorString((cudaError_t)e));
    }
    return S2D_OK;
}

int run_adjoint(Ctx *c, Batch &b, GradRun &g, StepArgs args, int kt_top, int n, int grid, bool use_graph,
                int *launches) {
    if (n <= 0) return S2D_OK;
    StepArgs *args_d = c->args_d.as<StepArgs>();
    const int chunk = use_graph ? std::max(1, c->opt_graph_chunk) : n;
    for (int done = 0; done < n; done += chunk) {
        const int m = std::min(chunk, n - done);
        args.kt_base = kt_top - done;
        int e = launch_set_args(args, args_d, c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "set_args launch: %s", cudaGetErrorString((cudaError_t)e));
        *launches += 1 + m;
        if (!use_graph) {
            for (int k = 0; k < m; ++k) {
                e = launch_adjoint(args_d, k, grid, 128, c->opt_adj_minb, c->stream);
                if (e) return fail(c, S2D_ERR_CUDA, "adjoint launch: %s", cudaGetErrorString((cudaError_t)e));
            }
            continue;
        }
        (void)g;
        const std::vector<long> key = {m, grid, c->opt_adj_minb};
        auto it = c->adj_graphs.find(key);
        if (it == c->adj_graphs.end()) {
            cudaGraph_t gr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < m; ++k) {
                e = launch_adjoint(args_d, k, grid, 128, c->opt_adj_minb, c->stream);
                if (e) {
                    cudaStreamEndCapture(c->stream, &gr);
                    if (gr) cudaGraphDestroy(gr);
                    return fail(c, S2D_ERR_CUDA, "adjoint capture: %s", cudaGetErrorString((cudaError_t)e));
                }
            }
            CK(cudaStreamEndCapture(c->stream, &gr));
            cudaGraphExec_t ge;
            cudaError_t ce = cudaGraphInstantiate(&ge, gr, 0);
            cudaGraphDestroy(gr);
            CK(ce);
            it = c->adj_graphs.emplace(key, ge).first;
        }
        CK(cudaGraphLaunch(it->second, c->stream));
    }
    return S2D_OK;
}

}  // namespace

extern "C" int s2d_gradient(void *ctx, const s2d_shot *shots, int nshots, const s2d_wave *wave,
                            const double *wavelet, int nwavelet, const float *data, float *grad_vp,
                            float *grad_rho, float *seis_out, double *misfit, double *grad_wavelet,
                            unsigned flags, s2d_stats *stats) {
    Ctx *c = static_cast<Ctx *>(ctx);
    if (!c) return S2D_ERR_ARG;
    if (!shots || nshots < 1 || !wave || !data || !grad_vp || !grad_rho)
        return fail(c, S2D_ERR_ARG, "null argument");
    for (int s = 1; s < nshots; ++s)
        if (shots[s].model_id != shots[0].model_id)
            return fail(c, S2D_ERR_ARG, "all shots of a gradient call must use one model");
    if (!(wave->fd_dt > 0) || !(wave->real_dt > 0) || !(wave->rec_len > 0) || !(wave->dom_freq > 0))
        return fail(c, S2D_ERR_ARG, "wave parameters must be positive");
    CK(cudaSetDevice(c->device));
    const bool dev_seis = (flags & S2D_SEIS_DEVICE) != 0;
    const bool dev_grad = (flags & S2D_GRAD_DEVICE) != 0;
    const bool use_graph = !(flags & S2D_NO_GRAPH);
    // forward batch: record into the caller's device buffer when there is one
    unsigned fflags = (dev_seis && seis_out) ? S2D_SEIS_DEVICE : 0u;
    {
        int e = setup_batch(c, shots, nshots, *wave, wavelet, nwavelet, seis_out, fflags);
        if (e) {
            c->drop_batch();
            return e;
        }
    }
    Batch &b = *c->batch;
    const RunSteps rs = b.steps;
    Model &m = *c->models[shots[0].model_id];
    const size_t F = m.field_elems, fb = F * sizeof(float);
    GradRun g;
    CK(cudaEventRecord(c->ev0, c->stream));
    int launches = 0;

    // per-shot adjoint state and source-adjoint trace; one accumulator pair
    // dJ/dkappa, dJ/db shared by every shot (they share the model): the
    // adjoint kernels add into it atomically
    std::vector<ShotDev> adj = b.shot_dev;
    std::vector<float *> gk(nshots), gb(nshots), sadj(nshots);
    float *acc_pair = nullptr;
    {
        void *p;
        int e = grad_alloc(c, g, 2 * fb, &p);
        if (e) return e;
        CK(cudaMemsetAsync(p, 0, 2 * fb, c->stream));
        acc_pair = static_cast<float *>(p);
    }
    for (int s = 0; s < nshots; ++s) {
        // adjoint state: 8 fields in one allocation, as the forward state
        void *p;
        {
            int e = grad_alloc(c, g, 8 * fb, &p);
            if (e) return e;
            CK(cudaMemsetAsync(p, 0, 8 * fb, c->stream));
            for (int par = 0; par < 2; ++par)
                for (int f = 0; f < 4; ++f) adj[s].st[par][f] = static_cast<float *>(p) + (size_t)(par * 4 + f) * F;
        }
        adj[s].grad[0] = acc_pair;
        adj[s].grad[1] = acc_pair + F;
        gk[s] = adj[s].grad[0];
        gb[s] = adj[s].grad[1];
        // 8th-order cell-parallel adjoint: two scratch fields for its velocity
        // gathers (ghosts stay 0); the streaming form keeps them in shared memory
        if (b.order8 && c->opt_adj8_form == 1) {
            int e = grad_alloc(c, g, 2 * fb, &p);
            if (e) return e;
            CK(cudaMemsetAsync(p, 0, 2 * fb, c->stream));
            adj[s].scr = static_cast<float *>(p);
        }
        int e = grad_alloc(c, g, sizeof(float) * rs.fd_nt, &p);
        if (e) return e;
        CK(cudaMemsetAsync(p, 0, sizeof(float) * rs.fd_nt, c->stream));
        sadj[s] = static_cast<float *>(p);
        adj[s].srcadj = sadj[s];
    }
    // adjoint source: the caller's, or the residual d - d_obs after the forward
    const size_t nseis = b.seis_elems;
    float *adj_src = nullptr;
    {
        void *p;
        int e = grad_alloc(c, g, std::max<size_t>(nseis, 1) * sizeof(float), &p);
        if (e) return e;
        adj_src = static_cast<float *>(p);
    }
    // checkpoint interval: the longest whose products and checkpoints fit in
    // free memory (pooled buffers count as free: the pool releases itself when
    // an allocation fails)
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    const double budget = 0.85 * ((double)free_b + (double)c->pool.held()) - 4.0 * fb - 64e6;
    const double per_step_all = (double)nshots * 4.0 * fb;
    auto need = [&](int C) { return per_step_all * (C + (rs.fd_nt + C - 1) / C - 1); };
    int C = -1;
    const int cmax = c->opt_grad_segment > 0 ? std::min(rs.fd_nt, c->opt_grad_segment) : rs.fd_nt;
    for (int t = cmax; t >= 1; --t)
        if (need(t) <= budget) {
            C = t;
            break;
        }
    if (C < 1) {
        int best = 1;
        for (int t = 1; t <= rs.fd_nt; ++t)
            if (need(t) < need(best)) best = t;
        return fail(c, S2D_ERR_NOMEM,
                    "gradient of %d shots needs at least %.1f GB for checkpoints and step products, %.1f GB "
                    "available; use fewer shots per call",
                    nshots, need(best) / 1e9, budget / 1e9);
    }
    const int nseg = (rs.fd_nt + C - 1) / C;
    std::vector<float *> prod(nshots), ckpt(nshots);
    for (int s = 0; s < nshots; ++s) {
        void *p;
        int e = grad_alloc(c, g, (size_t)C * 4 * fb, &p);
        if (e) return e;
        // ghost rows and the second product slot of merged cells are never
        // written; the adjoint reads them (times zero): they must hold zeros
        CK(cudaMemsetAsync(p, 0, (size_t)C * 4 * fb, c->stream));
        prod[s] = static_cast<float *>(p);
        ckpt[s] = nullptr;
        if (nseg > 1) {
            e = grad_alloc(c, g, (size_t)(nseg - 1) * 4 * fb, &p);
            if (e) return e;
            ckpt[s] = static_cast<float *>(p);
        }
        adj[s].prod = prod[s];
        adj[s].nprod = (size_t)C * 4 * F;
        adj[s].seis = adj_src + b.shots[s].seis_off;
        b.shot_dev[s].prod = prod[s];
        b.shot_dev[s].nprod = (size_t)C * 4 * F;
    }
    DevBuf adj_table;
    CK(adj_table.alloc(sizeof(ShotDev) * nshots));
    CK(cudaMemcpyAsync(adj_table.p, adj.data(), sizeof(ShotDev) * nshots, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(b.shots_d.p, b.shot_dev.data(), sizeof(ShotDev) * nshots, cudaMemcpyHostToDevice,
                       c->stream));

    LaunchCfg lc_fwd, lc_prod;
    const int prod_variant = b.order8 ? kVariantO8Products : c->opt_prod_variant;
    {
        int e = base_config(c, b, &lc_fwd);
        const int order = lc_fwd.order;
        // the gradient keeps every step's state (checkpoints at kt parity):
        // one step per launch
        if (!e && steps_per_launch(lc_fwd.variant) != 1)
            e = launch_config(c, b.max_tasks, &lc_fwd, kVariantLdgPf4, 128, 0);
        if (!e) e = layout_groups(c, b, lc_fwd);
        if (!e) e = launch_config(c, b.max_tasks, &lc_fwd, lc_fwd.variant, lc_fwd.block, lc_fwd.stages);
        if (!e) e = launch_config(c, b.max_tasks, &lc_prod, prod_variant, 128, 0);
        if (e) return e;
        lc_fwd.order = steps_per_launch(lc_fwd.variant) == 1 ? order : -1;
    }
    StepArgs fa{};
    fa.shots = b.shots_d.as<ShotDev>();
    fa.tmaps = b.tmaps_d.p;
    fa.tmap_mat0 = b.nshots;
    fa.groups = b.groups_d.as<GroupDev>();
    fa.ngroups = (int)b.groups.size();
    fa.total_tasks = batch_tasks(b);
    fa.dt_factor = rs.dt_factor;
    fa.fd_nt = rs.fd_nt;
    bool graph_used = false;
    {
        int e = phase_mark(c, g, kPhaseSweep);
        if (e) return e;
    }
    // ---- forward sweep, saving the state at each segment start ----
    auto save_ckpt = [&](int j) -> int {
        const int par = (j * C) & 1;
        for (int s = 0; s < nshots; ++s)
            for (int f = 0; f < 4; ++f)
                CK(cudaMemcpyAsync(ckpt[s] + ((size_t)j * 4 + f) * F, b.shot_dev[s].st[par][f], fb,
                                   cudaMemcpyDeviceToDevice, c->stream));
        return S2D_OK;
    };
    // The steps that keep their products (the last segment of the sweep, the
    // recomputes) and the adjoint steps run with a task layout for the
    // resident warps of the adjoint kernel: the two kernels of the backward
    // phase then each take whole rounds of tasks.
    int agrid = 1;
    auto backward_layout = [&]() -> int {
        if (b.order8) {
            // the 8th-order products kernel and the streaming adjoint share the
            // 112-row layout (the cell-parallel adjoint needs none)
            int e = layout_groups(c, b, lc_prod);
            if (!e) e = launch_config(c, b.max_tasks, &lc_prod, prod_variant, 128, 0);
            fa.total_tasks = batch_tasks(b);
            return e;
        }
        int bps = 0;
        if (adjoint_kernel_occupancy(128, c->opt_adj_minb, &bps) || bps < 1) bps = 1;
        const long resident = (long)c->sm_count * bps;
        int e = layout_groups_for(c, b, resident * 4, {-1, resident, c->opt_seg_len});
        if (!e) e = launch_config(c, b.max_tasks, &lc_prod, c->opt_prod_variant, 128, 0);
        if (e) return e;
        agrid = (int)std::max<long>(1, std::min<long>(resident, (b.max_tasks * 32 + 127) / 128));
        fa.total_tasks = batch_tasks(b);
        return S2D_OK;
    };
    for (int j = 0; j < nseg; ++j) {
        const int k0 = j * C, n = std::min(C, rs.fd_nt - k0);
        b.cur = k0 & 1;  // one step per launch: the state of step kt is in buffer kt & 1
        if (j < nseg - 1) {
            StepArgs a = fa;
            int e = save_ckpt(j);
            if (!e) e = run_loop(c, b, lc_fwd, a, k0, n, use_graph, &launches, &graph_used);
            if (e) return e;
        } else {
            int e = backward_layout();
            if (e) return e;
            StepArgs a = fa;
            a.flags = S2D_STEP_PRODUCTS;
            a.prod_kt0 = k0;
            e = run_loop(c, b, lc_prod, a, k0, n, use_graph, &launches, &graph_used);
            if (e) return e;
        }
    }
    // ---- adjoint source ----
    {
        int e = phase_mark(c, g, kPhaseOther);
        if (e) return e;
    }
    DevBuf sumsq;
    CK(sumsq.alloc(sizeof(double)));
    CK(cudaMemsetAsync(sumsq.p, 0, sizeof(double), c->stream));
    const cudaMemcpyKind dk = dev_seis ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (flags & S2D_GRAD_MISFIT) {
        const float *obs = data;
        if (!dev_seis) {
            CK(cudaMemcpyAsync(adj_src, data, nseis * sizeof(float), cudaMemcpyHostToDevice, c->stream));
            obs = adj_src;
        }
        int e = launch_residual(b.seis_d, obs, adj_src, nseis, sumsq.as<double>(), c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "residual launch: %s", cudaGetErrorString((cudaError_t)e));
    } else {
        CK(cudaMemcpyAsync(adj_src, data, nseis * sizeof(float), dk, c->stream));
    }
    // ---- backward over the segments ----
    StepArgs aa = fa;
    // the adjoint's warps of a block take one tile of consecutive shots (task
    // order 0): measured 1.5% faster than order 1 on the c5 gradient
    aa.task_order = 0;
    aa.shots = adj_table.as<ShotDev>();
    aa.err = c->dev_err.as<int>();
    for (int j = nseg - 1; j >= 0; --j) {
        const int k0 = j * C, n = std::min(C, rs.fd_nt - k0);
        if (j < nseg - 1) {
            int e = phase_mark(c, g, kPhaseRecompute);
            if (e) return e;
            const int par = k0 & 1;
            for (int s = 0; s < nshots; ++s)
                for (int f = 0; f < 4; ++f)
                    CK(cudaMemcpyAsync(b.shot_dev[s].st[par][f], ckpt[s] + ((size_t)j * 4 + f) * F, fb,
                                       cudaMemcpyDeviceToDevice, c->stream));
            StepArgs a = fa;
            a.flags = S2D_STEP_PRODUCTS | S2D_STEP_NO_RECORD;
            a.prod_kt0 = k0;
            b.cur = k0 & 1;
            e = run_loop(c, b, lc_prod, a, k0, n, use_graph, &launches, &graph_used);
            if (e) return e;
        }
        StepArgs a = aa;
        a.prod_kt0 = k0;
        int e = phase_mark(c, g, kPhaseAdjoint);
        if (e) return e;
        e = b.order8 ? run_adjoint8(c, a, k0 + n - 1, n, m.nnx, m.nnz, nshots, &launches)
                         : run_adjoint(c, b, g, a, k0 + n - 1, n, agrid, use_graph, &launches);
        if (e) return e;
    }
    // ---- source term, chain rule, fold ----
    {
        int e = phase_mark(c, g, kPhaseOther);
        if (e) return e;
    }
    std::vector<double> wv;
    int inject_last;
    if (wavelet) {
        wv.assign(wavelet, wavelet + std::max(nwavelet, 0));
        inject_last = nwavelet - 1;
    } else {
        wv = ricker(*wave, rs.nts);
        inject_last = rs.nts;
    }
    std::vector<float> sa(rs.fd_nt);
    std::vector<int> cells(nshots);
    std::vector<double> vals(nshots);
    const double sfac = (double)wave->fd_dt / (double)(m.dx * m.dz);
    for (int s = 0; s < nshots; ++s) {
        CK(cudaMemcpyAsync(sa.data(), sadj[s], sizeof(float) * rs.fd_nt, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        // kappa at the source, in double as the amplitude uses it (cpumodelling.cpp:136-140)
        const int mx = std::min(std::max(b.shots[s].src_x - m.nb, 0), m.nx - 1);
        const int mz = std::min(std::max(b.shots[s].src_z - m.nb, 0), m.nz - 1);
        float vr[2];
        CK(cudaMemcpy(&vr[0], m.vp.as<float>() + (size_t)mx * m.nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&vr[1], m.rho.as<float>() + (size_t)mx * m.nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
        const double ksrc = m.free_surface && b.shots[s].src_z <= m.nb
                                ? 0.0
                                : ((double)vr[0] * (double)vr[0]) * (double)vr[1];
        double v = 0;
        for (int kt = 0; kt < rs.fd_nt; ++kt) {
            const bool injected = kt <= inject_last;
            const double wk = injected && kt < (int)wv.size() ? wv[kt] : 0.0;
            if (injected) v += (double)sa[kt] * (wave->fd_dt * wk / (double)(m.dx * m.dz));
            if (grad_wavelet)
                grad_wavelet[(size_t)s * rs.fd_nt + kt] = injected ? (double)sa[kt] * sfac * ksrc : 0.0;
        }
        vals[s] = v;
        cells[s] = (int)((size_t)(b.shots[s].src_x + S2D_GX) * m.ld + (b.shots[s].src_z + S2D_GZ));
    }
    void *p_cells, *p_vals, *p_ptrs, *p_tmp, *p_pad, *p_out = nullptr;
    {
        int e = grad_alloc(c, g, sizeof(int) * nshots, &p_cells);
        if (!e) e = grad_alloc(c, g, sizeof(double) * nshots, &p_vals);
        if (!e) e = grad_alloc(c, g, sizeof(float *) * 2 * nshots, &p_ptrs);
        if (!e) e = grad_alloc(c, g, 2 * fb, &p_tmp);
        if (!e) e = grad_alloc(c, g, 2 * fb, &p_pad);
        if (!e && !dev_grad) e = grad_alloc(c, g, 2 * sizeof(float) * m.nx * m.nz, &p_out);
        if (e) return e;
    }
    std::vector<float *> ptrs;
    ptrs.insert(ptrs.end(), gk.begin(), gk.end());
    ptrs.insert(ptrs.end(), gb.begin(), gb.end());
    CK(cudaMemcpyAsync(p_cells, cells.data(), sizeof(int) * nshots, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(p_vals, vals.data(), sizeof(double) * nshots, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(p_ptrs, ptrs.data(), sizeof(float *) * 2 * nshots, cudaMemcpyHostToDevice, c->stream));
    float **dptrs = static_cast<float **>(p_ptrs);
    float *out_vp = dev_grad ? grad_vp : static_cast<float *>(p_out);
    float *out_rho = dev_grad ? grad_rho : static_cast<float *>(p_out) + (size_t)m.nx * m.nz;
    {
        int e = launch_gradient_finalize(dptrs, dptrs + nshots, nshots, 1,
                                         static_cast<int *>(p_cells), static_cast<double *>(p_vals),
                                         m.vp.as<float>(), m.rho.as<float>(), m.nx, m.nz, m.nb, m.ld,
                                         m.free_surface ? m.nb + 1 : 0,
                                         static_cast<float *>(p_tmp), static_cast<float *>(p_pad),
                                         static_cast<float *>(p_pad) + F, out_vp, out_rho, c->stream);
        if (e) return fail(c, S2D_ERR_CUDA, "gradient finalize: %s", cudaGetErrorString((cudaError_t)e));
    }
    launches += 5;
    CK(cudaEventRecord(c->ev1, c->stream));
    if (!dev_grad) {
        CK(cudaMemcpyAsync(grad_vp, out_vp, sizeof(float) * m.nx * m.nz, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(grad_rho, out_rho, sizeof(float) * m.nx * m.nz, cudaMemcpyDeviceToHost, c->stream));
    }
    if (seis_out && !(fflags & S2D_SEIS_DEVICE))
        CK(cudaMemcpyAsync(seis_out, b.seis_d, nseis * sizeof(float),
                           dev_seis ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
    double ss = 0;
    CK(cudaMemcpyAsync(&ss, sumsq.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (misfit) *misfit = 0.5 * ss;
    // the forward state buffers now hold recomputed states: no continuation
    b.kt_next = -1;
    {
        int e = check_device_error(c);
        if (e) return e;
    }
    for (auto &bp : g.bufs) c->pool.give(std::move(bp));
    g.bufs.clear();
    if (stats) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        stats->loop_ms = ms;
        stats->cell_updates = (double)m.nnx * m.nnz * nshots * rs.fd_nt;
        stats->gcells_per_s = ms > 0 ? stats->cell_updates / (ms * 1e6) : 0.0;
        stats->kernel_launches = launches;
        stats->graph_used = graph_used ? 1 : 0;
        stats->grad_segment = C;
        double ph[4] = {0, 0, 0, 0};
        for (size_t i = 0; i < g.marks.size(); ++i) {
            cudaEvent_t end = i + 1 < g.marks.size() ? c->phase_ev[g.marks[i + 1].second] : c->ev1;
            float t = 0;
            CK(cudaEventElapsedTime(&t, c->phase_ev[g.marks[i].second], end));
            ph[g.marks[i].first] += t;
        }
        stats->task_order = lc_fwd.order >= 0 ? lc_fwd.order : c->opt_order;
        stats->sweep_ms = ph[kPhaseSweep];
        stats->recompute_ms = ph[kPhaseRecompute];
        stats->adjoint_ms = ph[kPhaseAdjoint];
    }
    c->last_segment = C;
    return S2D_OK;
}

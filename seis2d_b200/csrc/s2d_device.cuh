// Device helpers shared by the forward and adjoint step kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "s2d_internal.h"

namespace s2d {

static constexpr unsigned kFull = 0xffffffffu;

static __device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
static __device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
// p[0..3] += v as one vector reduction in L2 (red: no value comes back, so
// the warp does not wait for it; p 16-byte aligned).
static __device__ __forceinline__ void red_add4(float *p, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
// Copies a shot record into this warp's shared-memory slot (every lane
// takes part; nothing may read the slot meanwhile).  Loops that re-read the
// record's pointers and constants then read shared memory, not L1, where the
// streamed columns evict them.
static __device__ __forceinline__ void warp_copy_shot(ShotDev &dst, const ShotDev &src, int lane) {
    static_assert(sizeof(ShotDev) % 8 == 0, "shot record copied in 8-byte words");
    __syncwarp();
    for (int i = lane; i < (int)(sizeof(ShotDev) / 8); i += 32)
        reinterpret_cast<unsigned long long *>(&dst)[i] = reinterpret_cast<const unsigned long long *>(&src)[i];
    __syncwarp();
}
static __device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// 16-byte asynchronous copy global -> shared (cp.async, L2 only); read =
// false copies nothing and zero-fills the 16 bytes.
static __device__ __forceinline__ void cp_async16(void *dst, const void *src, bool read) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(read ? 16 : 0)
                 : "memory");
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
static __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Coefficients (c0, c1) of a0*(f[i]-f[i-1]) + a1*(f[i+1]-f[i-2]) per row of
// the backward operators: 4th order on rows [2, n-2], plain difference on
// rows 1 and n-1, zero on row 0 and outside the grid
// (cpu_modelling_kernels.cpp:201-258).
static __device__ __forceinline__ void dm_coef(int i, int n, float &c0, float &c1) {
    if (i >= 2 && i <= n - 2) { c0 = kA0; c1 = kA1; }
    else if (i == 1 || i == n - 1) { c0 = 1.0f; c1 = 0.0f; }
    else { c0 = 0.0f; c1 = 0.0f; }
}
// Forward operators a0*(f[i+1]-f[i]) + a1*(f[i+2]-f[i-1]): 4th order on rows
// [1, n-3], plain difference on rows 0 and n-2, zero on row n-1
// (cpu_modelling_kernels.cpp:260-316).
static __device__ __forceinline__ void dp_coef(int i, int n, float &c0, float &c1) {
    if (i >= 1 && i <= n - 3) { c0 = kA0; c1 = kA1; }
    else if (i == 0 || i == n - 2) { c0 = 1.0f; c1 = 0.0f; }
    else { c0 = 0.0f; c1 = 0.0f; }
}

// 8th-order staggered coefficients (1225/1024, -245/3072, 49/5120, -5/7168 in
// float) and the coefficients of row i of the 8th-order D- (taps i-4 .. i+3,
// f[i+k] - f[i-1-k] for k = 0..3) and D+ (taps i-3 .. i+4, f[i+1+k] - f[i-k]):
// the reference's pairs (a0, a1), (1, 0) or 0 where the 8 taps would leave the
// grid.
constexpr float kC81 = 1225.0f / 1024.0f;
constexpr float kC82 = -245.0f / 3072.0f;
constexpr float kC83 = 49.0f / 5120.0f;
constexpr float kC84 = -5.0f / 7168.0f;
static __device__ __forceinline__ float4 dm8(int i, int n) {
    if (i >= 4 && i <= n - 4) return make_float4(kC81, kC82, kC83, kC84);
    float c0, c1;
    dm_coef(i, n, c0, c1);
    return make_float4(c0, c1, 0.0f, 0.0f);
}
static __device__ __forceinline__ float4 dp8(int i, int n) {
    if (i >= 3 && i <= n - 5) return make_float4(kC81, kC82, kC83, kC84);
    float c0, c1;
    dp_coef(i, n, c0, c1);
    return make_float4(c0, c1, 0.0f, 0.0f);
}

static __device__ __forceinline__ float comp(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// Per-lane constants of one task.  FAST tasks lie inside the shot's fast row
// range (no z-sponge, no edge rows): their row coefficients are literals.
// Other tasks read a row's coefficients when they use them (L1 hits), so that
// neither kind holds per-row tables in registers.
template <bool FAST>
struct Lane {
    int z0;          // first row of the lane
    int zl;          // row the lane's loads start at: z0, or -S2D_GZ for a ghost lane
    bool owner;      // writes its rows (lanes 1..30 whose rows are in the grid)
    int sdz;         // source row - z0
    int src_x;       // source column
    float amp;       // source term of this step
    float kz;        // interior kz (FAST)
    float kx;        // interior kx (x-interior columns)
    int nnz;
    const float4 *zc;  // zcoef + z0 + GZ (not FAST)
};

template <bool FAST>
static __device__ __forceinline__ void lane_setup(Lane<FAST> &ln, const ShotDev &S, int c, int lane, int kt) {
    ln.z0 = c + S2D_ZPT * lane;
    // A ghost lane (all 4 rows above or below the grid: the first lane of the
    // first strip, the lanes of the last strip past nnz) holds only ghost
    // cells, which are zero and stay zero.  It loads the column's first ghost
    // row instead (zeros: one 16-byte piece shared by all such lanes of a warp
    // instead of DRAM traffic of its own) and writes nothing.
    const bool ghost = ln.z0 < 0 || ln.z0 >= S.nnz;
    ln.zl = ghost ? -S2D_GZ : ln.z0;
    ln.owner = lane >= 1 && lane <= 30 && !ghost;
    ln.sdz = S.src_z - ln.z0;
    ln.src_x = S.src_x;
    ln.amp = __ldg(S.amp + kt);
    ln.kz = S.kz_in;
    ln.kx = S.kx_in;
    ln.nnz = S.nnz;
    ln.zc = S.zcoef + (ln.z0 + S2D_GZ);
}

// damp1a, kz*damp1a1, damp1b, kz*damp1b1 of the lane's row z0 + i
template <bool FAST>
static __device__ __forceinline__ float4 zrow(const Lane<FAST> &ln, int i) {
    if (FAST) return make_float4(1.0f, ln.kz, 1.0f, ln.kz);
    return __ldg(ln.zc + i);
}
// operator pairs of the lane's row z0 + i (D- and D+)
template <bool FAST>
static __device__ __forceinline__ void zdm(const Lane<FAST> &ln, int i, float &c0, float &c1) {
    if (FAST) { c0 = kA0; c1 = kA1; return; }
    dm_coef(ln.z0 + i, ln.nnz, c0, c1);
}
template <bool FAST>
static __device__ __forceinline__ void zdp(const Lane<FAST> &ln, int i, float &c0, float &c1) {
    if (FAST) { c0 = kA0; c1 = kA1; return; }
    dp_coef(ln.z0 + i, ln.nnz, c0, c1);
}

// Rows [lo, hi] of a task all in the shot's fast range.
static __device__ __forceinline__ bool rows_fast(const ShotDev &S, int lo, int hi) {
    return lo >= S.zfast_lo && hi < S.zfast_hi;
}

// Map a flat task index to (shot, strip, first column, segment length).
// Order 0 runs the shots of one (strip, segment) on consecutive warps, so they
// share that tile of the model through L2.  Order 1 runs the strips of one
// (shot, segment) on consecutive warps, so the warps of a block read adjacent
// pieces of each column (contiguous DRAM rows); the shots of one segment still
// run close together and share the segment's materials in L2.
static __device__ __forceinline__ const ShotDev &task_of(const StepArgs &a, int t, int &strip, int &xa, int &seg_len) {
    int g = 0;
    while (g + 1 < a.ngroups && __ldg(&a.groups[g + 1].task_begin) <= t) ++g;
    const GroupDev &G = a.groups[g];
    int tl = t - G.task_begin;
    int s;
    if (a.task_order == 0) {
        s = G.shot0 + tl % G.nshots;
        tl /= G.nshots;
        strip = tl % G.nstrips;
        xa = (tl / G.nstrips) * G.seg_len;
    } else {
        strip = tl % G.nstrips;
        tl /= G.nstrips;
        s = G.shot0 + tl % G.nshots;
        xa = (tl / G.nshots) * G.seg_len;
    }
    seg_len = G.seg_len;
    return a.shots[s];
}


// Debug self-check (built with -DS2D_DEVICE_CHECKS): the ranges every access
// of one task touches, from the runtime tables.  A failed check records a
// code in the error word and the task is skipped.
static __device__ __forceinline__ bool task_in_bounds(const StepArgs &a, const ShotDev &S, int strip, int xa,
                                                      int seg_len, int kt, bool prod, int code) {
#ifdef S2D_DEVICE_CHECKS
    const size_t ld = (size_t)S.ld;
    const int xb = min(S.nnx, xa + seg_len);
    const size_t F = (size_t)(S.nnx + 2 * S2D_GX) * ld;
    const long c = (long)strip * S2D_STRIP_OUT - 4;
    const long lo = (long)(xa - 3 + S2D_GX) * (long)ld + (c + S2D_GZ);
    const long hi = (long)(xb + 2 + S2D_GX) * (long)ld + (c + S2D_GZ) + 127;
    int bad = 0;
    if (ld % 4 || (c + S2D_GZ) % 4) bad = 1;
    else if (F > S.nfield) bad = 2;
    else if (lo < 0 || hi >= (long)F) bad = 3;
    else if (c + 127 + S2D_GZ >= (long)ld) bad = 4;
    else if (kt < 0 || kt >= a.fd_nt) bad = 5;
    else if (prod && ((long)(kt - a.prod_kt0) < 0 || (size_t)(kt - a.prod_kt0 + 1) * 4 * F > S.nprod)) bad = 6;
    else if ((size_t)S.nrec * S.real_nt > S.nseis) bad = 7;
    else if (S.src_x < 0 || S.src_x >= S.nnx || S.src_z < 0 || S.src_z >= S.nnz) bad = 8;
    if (bad) {
        if (a.err) atomicCAS(a.err, 0, (code << 8) | bad);
        return false;
    }
#endif
    return true;
}

}  // namespace s2d

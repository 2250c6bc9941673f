// FD time-step kernels of libseis2d for sm_100a.
//
// One launch advances every shot of a batch by one FD step of the scheme in
// src/src_cpu/cpumodelling.cpp:115-156 (FDOperator_4): D-x vx, D-z vz, the
// split-field pressure update with sponge, source injection, p = px + pz,
// D+x p, D+z p and the particle-velocity update with sponge, plus receiver
// sampling of p (cpumodelling.cpp:356-360).  All of it is fused into one pass:
//
//   * A warp owns a strip of 128 rows (each lane 4 consecutive z rows, one
//     float4) and streams along x over a segment of columns.  It keeps
//     sliding windows of vx (4 columns), new p (4 columns) and vz (3 columns)
//     in registers, so every field is read from HBM once per step, and the
//     x-stencils need no shared memory.
//   * z-neighbours come from the adjacent lanes by warp shuffles.  The strip
//     overlaps its neighbours by 4 rows on each side and writes only the
//     middle 120 rows, so warps never exchange data and never synchronise.
//   * State is double-buffered (read parity kt&1, write the other), which is
//     what lets pressure and velocity of one step share a single pass.
//
// Traffic per cell-update: px, pz, vx, vz read once and written once
// (32 B) and kappa, bx, bz read once (12 B, shared through L2 by the shots
// of a batch that use the same model).
#include <cuda_runtime.h>

#include "s2d_internal.h"

namespace s2d {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

// Coefficients (c0, c1) of a0*(f[i]-f[i-1]) + a1*(f[i+1]-f[i-2]) per row of
// the backward operators: 4th order on rows [2, n-2], plain difference on
// rows 1 and n-1, zero on row 0 and outside the grid
// (cpu_modelling_kernels.cpp:201-258).
__device__ __forceinline__ void dm_coef(int i, int n, float &c0, float &c1) {
    if (i >= 2 && i <= n - 2) { c0 = kA0; c1 = kA1; }
    else if (i == 1 || i == n - 1) { c0 = 1.0f; c1 = 0.0f; }
    else { c0 = 0.0f; c1 = 0.0f; }
}
// Forward operators a0*(f[i+1]-f[i]) + a1*(f[i+2]-f[i-1]): 4th order on rows
// [1, n-3], plain difference on rows 0 and n-2, zero on row n-1
// (cpu_modelling_kernels.cpp:260-316).
__device__ __forceinline__ void dp_coef(int i, int n, float &c0, float &c1) {
    if (i >= 1 && i <= n - 3) { c0 = kA0; c1 = kA1; }
    else if (i == 0 || i == n - 2) { c0 = 1.0f; c1 = 0.0f; }
    else { c0 = 0.0f; c1 = 0.0f; }
}

__device__ __forceinline__ float comp(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// One (shot, strip, x-segment) task of one FD step.
__device__ __forceinline__ void run_task(const ShotDev &S, int strip, int xa, int seg_len, int kt,
                                         int par, bool rec, int slot, int lane) {
    const int nnx = S.nnx, nnz = S.nnz;
    const size_t ld = (size_t)S.ld;
    const int xb = min(nnx, xa + seg_len);
    const int c = strip * S2D_STRIP_OUT - 4;  // first row the warp reads
    const int z0 = c + S2D_ZPT * lane;         // first row of this lane
    const size_t off = (size_t)(z0 + S2D_GZ) + (size_t)S2D_GX * ld;

    const float *__restrict__ pxi = S.st[par][0] + off;
    const float *__restrict__ pzi = S.st[par][1] + off;
    const float *__restrict__ vxi = S.st[par][2] + off;
    const float *__restrict__ vzi = S.st[par][3] + off;
    float *__restrict__ pxo = S.st[par ^ 1][0] + off;
    float *__restrict__ pzo = S.st[par ^ 1][1] + off;
    float *__restrict__ vxo = S.st[par ^ 1][2] + off;
    float *__restrict__ vzo = S.st[par ^ 1][3] + off;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = S.bx + off;
    const float *__restrict__ bzp = S.bz + off;

    // Row constants of this lane's four rows.
    const float4 *zc = S.zcoef + (z0 + S2D_GZ);
    const float4 zc0 = __ldg(zc + 0), zc1 = __ldg(zc + 1), zc2 = __ldg(zc + 2), zc3 = __ldg(zc + 3);
    float cm0[4], cm1[4], cp0[4], cp1[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        dm_coef(z0 + i, nnz, cm0[i], cm1[i]);
        dp_coef(z0 + i, nnz, cp0[i], cp1[i]);
    }
    const bool owner = lane >= 1 && lane <= 30;  // rows [c+4, c+124)
    const int sdz = S.src_z - z0;
    const float amp = __ldg(S.amp + kt);
    const bool src_lane = sdz >= 0 && sdz < 4;

    float4 vq0, vq1, vq2, vq3;  // vx at columns L-3 .. L
    float4 pq0, pq1, pq2, pq3;  // new p at columns L-4 .. L-1
    float4 zq0, zq1, zq2;       // old vz at columns L-3 .. L-1
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    vq1 = ld4(vxi + (ptrdiff_t)(xa - 3) * (ptrdiff_t)ld);
    vq2 = ld4(vxi + (ptrdiff_t)(xa - 2) * (ptrdiff_t)ld);
    vq3 = ld4(vxi + (ptrdiff_t)(xa - 1) * (ptrdiff_t)ld);
    vq0 = zero;
    pq1 = pq2 = pq3 = zero;
    zq1 = zq2 = zero;

    for (int L = xa; L <= xb + 2; ++L) {
        // ---- pressure at column P = L - 1 (p computed on [xa-1, xb+1]) ----
        const int P = L - 1;
        const ptrdiff_t colL = (ptrdiff_t)L * (ptrdiff_t)ld;
        const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
        vq0 = vq1; vq1 = vq2; vq2 = vq3;
        vq3 = ld4(vxi + colL);
        const float4 px = ld4(pxi + colP);
        const float4 pz = ld4(pzi + colP);
        const float4 kk = ld4(kap + colP);
        const float4 vz = ld4(vzi + colP);
        const float4 xcP = __ldg(S.xcoef + (P + S2D_GX));
        float cx0, cx1;
        dm_coef(P, nnx, cx0, cx1);

        const float vz_up_z = __shfl_up_sync(kFull, vz.z, 1);
        const float vz_up_w = __shfl_up_sync(kFull, vz.w, 1);
        const float vz_dn_x = __shfl_down_sync(kFull, vz.x, 1);
        const float dz0 = cm0[0] * (vz.x - vz_up_w) + cm1[0] * (vz.y - vz_up_z);
        const float dz1 = cm0[1] * (vz.y - vz.x) + cm1[1] * (vz.z - vz_up_w);
        const float dz2 = cm0[2] * (vz.z - vz.y) + cm1[2] * (vz.w - vz.x);
        const float dz3 = cm0[3] * (vz.w - vz.z) + cm1[3] * (vz_dn_x - vz.y);
        const float dx0 = cx0 * (vq2.x - vq1.x) + cx1 * (vq3.x - vq0.x);
        const float dx1 = cx0 * (vq2.y - vq1.y) + cx1 * (vq3.y - vq0.y);
        const float dx2 = cx0 * (vq2.z - vq1.z) + cx1 * (vq3.z - vq0.z);
        const float dx3 = cx0 * (vq2.w - vq1.w) + cx1 * (vq3.w - vq0.w);

        float4 pxn, pzn;
        pxn.x = xcP.x * px.x + (xcP.y * kk.x) * dx0;
        pxn.y = xcP.x * px.y + (xcP.y * kk.y) * dx1;
        pxn.z = xcP.x * px.z + (xcP.y * kk.z) * dx2;
        pxn.w = xcP.x * px.w + (xcP.y * kk.w) * dx3;
        pzn.x = zc0.x * pz.x + (zc0.y * kk.x) * dz0;
        pzn.y = zc1.x * pz.y + (zc1.y * kk.y) * dz1;
        pzn.z = zc2.x * pz.z + (zc2.y * kk.z) * dz2;
        pzn.w = zc3.x * pz.w + (zc3.y * kk.w) * dz3;
        if (P == S.src_x && src_lane) {  // cpumodelling.cpp:136-140
            if (sdz == 0) pxn.x += amp;
            else if (sdz == 1) pxn.y += amp;
            else if (sdz == 2) pxn.z += amp;
            else pxn.w += amp;
        }
        const float4 pn = make_float4(pxn.x + pzn.x, pxn.y + pzn.y, pxn.z + pzn.z, pxn.w + pzn.w);
        const bool in_seg_p = P >= xa && P < xb;
        if (in_seg_p && owner) {
            st4(pxo + colP, pxn);
            st4(pzo + colP, pzn);
        }
        if (rec && in_seg_p) {
            const int j1 = __ldg(S.rec_ptr + P + 1);
            for (int j = __ldg(S.rec_ptr + P); j < j1; ++j) {
                const int d = __ldg(S.rec_z + j) - z0;
                if (owner && d >= 0 && d < 4)
                    S.seis[(size_t)__ldg(S.rec_id + j) * S.real_nt + slot] = comp(pn, d);
            }
        }
        pq0 = pq1; pq1 = pq2; pq2 = pq3; pq3 = pn;
        zq0 = zq1; zq1 = zq2; zq2 = vz;

        // ---- velocity at column V = L - 3 ----
        if (L >= xa + 3) {
            const int V = L - 3;
            const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
            const float4 bx = ld4(bxp + colV);
            const float4 bz = ld4(bzp + colV);
            const float4 xcV = __ldg(S.xcoef + (V + S2D_GX));
            float ux0, ux1;
            dp_coef(V, nnx, ux0, ux1);
            const float ex0 = ux0 * (pq2.x - pq1.x) + ux1 * (pq3.x - pq0.x);
            const float ex1 = ux0 * (pq2.y - pq1.y) + ux1 * (pq3.y - pq0.y);
            const float ex2 = ux0 * (pq2.z - pq1.z) + ux1 * (pq3.z - pq0.z);
            const float ex3 = ux0 * (pq2.w - pq1.w) + ux1 * (pq3.w - pq0.w);
            const float4 q = pq1;
            const float q_up_w = __shfl_up_sync(kFull, q.w, 1);
            const float q_dn_x = __shfl_down_sync(kFull, q.x, 1);
            const float q_dn_y = __shfl_down_sync(kFull, q.y, 1);
            const float ez0 = cp0[0] * (q.y - q.x) + cp1[0] * (q.z - q_up_w);
            const float ez1 = cp0[1] * (q.z - q.y) + cp1[1] * (q.w - q.x);
            const float ez2 = cp0[2] * (q.w - q.z) + cp1[2] * (q_dn_x - q.y);
            const float ez3 = cp0[3] * (q_dn_x - q.w) + cp1[3] * (q_dn_y - q.z);
            float4 vxn, vzn;
            vxn.x = xcV.z * vq0.x + (xcV.w * bx.x) * ex0;
            vxn.y = xcV.z * vq0.y + (xcV.w * bx.y) * ex1;
            vxn.z = xcV.z * vq0.z + (xcV.w * bx.z) * ex2;
            vxn.w = xcV.z * vq0.w + (xcV.w * bx.w) * ex3;
            vzn.x = zc0.z * zq0.x + (zc0.w * bz.x) * ez0;
            vzn.y = zc1.z * zq0.y + (zc1.w * bz.y) * ez1;
            vzn.z = zc2.z * zq0.z + (zc2.w * bz.z) * ez2;
            vzn.w = zc3.z * zq0.w + (zc3.w * bz.w) * ez3;
            if (owner) {
                st4(vxo + colV, vxn);
                st4(vzo + colV, vzn);
            }
        }
    }
}

__global__ void __launch_bounds__(128) step_kernel(const StepArgs *__restrict__ A, int kt_off) {
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    const int par = kt & 1;
    const bool rec = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int g = 0;
        while (g + 1 < a.ngroups && __ldg(&a.groups[g + 1].task_begin) <= t) ++g;
        const GroupDev &G = a.groups[g];
        int tl = t - G.task_begin;
        const int s = G.shot0 + tl % G.nshots;
        tl /= G.nshots;
        const int strip = tl % G.nstrips;
        const int seg = tl / G.nstrips;
        const ShotDev &S = a.shots[s];
        run_task(S, strip, seg * G.seg_len, G.seg_len, kt, par, rec && slot < S.real_nt, slot, lane);
    }
}

// ---- model preparation (cpumodelling.cpp:207-230, cpu_modelling_kernels.cpp:64-121) ----

// kappa = vp^2 rho in double rounded to float, buoyancy 1/rho (1e10 where
// rho <= 0) of the model expanded into the sponge by edge replication.
__global__ void prepare_cells(const float *__restrict__ vp, const float *__restrict__ rho, int nx, int nz,
                              int nb, int nnx, int nnz, int ld, float *kappa, float *bue) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (z >= nnz || x >= nnx) return;
    const int sx = min(max(x - nb, 0), nx - 1);
    const int sz = min(max(z - nb, 0), nz - 1);
    const float v = vp[(size_t)sx * nz + sz];
    const float r = rho[(size_t)sx * nz + sz];
    const size_t id = (size_t)(x + S2D_GX) * ld + (z + S2D_GZ);
    const double v2 = (double)v * (double)v;
    kappa[id] = (float)(v2 * (double)r);
    bue[id] = r > 0.0f ? 1.0f / r : 10000000000.0f;
}

// Staggered buoyancies: bz = z-average (last row 0), bx = x-average (last
// column = bz of column nnx-2).
__global__ void prepare_staggered(const float *__restrict__ bue, int nnx, int nnz, int ld, float *bx,
                                  float *bz) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (z >= nnz || x >= nnx) return;
    const size_t id = (size_t)(x + S2D_GX) * ld + (z + S2D_GZ);
    const float bzv = z < nnz - 1 ? 0.5f * (bue[id + 1] + bue[id]) : 0.0f;
    bz[id] = bzv;
    float bxv;
    if (x < nnx - 1) {
        bxv = 0.5f * (bue[id + ld] + bue[id]);
    } else {
        const size_t il = id - ld;
        bxv = z < nnz - 1 ? 0.5f * (bue[il + 1] + bue[il]) : 0.0f;
    }
    bx[id] = bxv;
}

__global__ void set_args_kernel(StepArgs v, StepArgs *dst) { *dst = v; }

}  // namespace

int launch_step(const StepArgs *args_dev, int kt_off, int grid, int block, void *stream) {
    step_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    return (int)cudaGetLastError();
}

int launch_set_args(const StepArgs &v, StepArgs *args_dev, void *stream) {
    set_args_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(v, args_dev);
    return (int)cudaGetLastError();
}

int launch_prepare_model(const float *vp, const float *rho, int nx, int nz, int nb, int ld, float *kappa,
                         float *bue, float *bx, float *bz, void *stream) {
    const int nnx = nx + 2 * nb, nnz = nz + 2 * nb;
    dim3 blk(256), grd((nnz + 255) / 256, nnx);
    prepare_cells<<<grd, blk, 0, (cudaStream_t)stream>>>(vp, rho, nx, nz, nb, nnx, nnz, ld, kappa, bue);
    prepare_staggered<<<grd, blk, 0, (cudaStream_t)stream>>>(bue, nnx, nnz, ld, bx, bz);
    return (int)cudaGetLastError();
}

int step_kernel_occupancy(int block, int *blocks_per_sm) {
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel, block, 0);
}

int step_kernel_attributes(int *regs, int *local_bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, step_kernel);
    if (e != cudaSuccess) return (int)e;
    *regs = fa.numRegs;
    *local_bytes = (int)fa.localSizeBytes;
    return 0;
}

}  // namespace s2d

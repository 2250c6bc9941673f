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
//     in registers, so every field is read from HBM once per step and the
//     x-stencils need no shared-memory exchange.
//   * z-neighbours come from the adjacent lanes by warp shuffles.  The strip
//     overlaps its neighbours by 4 rows on each side and writes only the
//     middle 120 rows, so warps never exchange data and never synchronise.
//   * State is double-buffered (read parity kt&1, write the other), which is
//     what lets pressure and velocity of one step share a single pass.
//
// Two ways to bring the columns in:
//   kVariantBulk  each warp runs its own asynchronous pipeline: one lane issues
//                 cp.async.bulk copies (TMA engine) of the 512-byte column
//                 pieces `stages` iterations ahead into a shared-memory ring,
//                 completion tracked by one mbarrier per stage (transaction
//                 bytes).  Loads need no registers while in flight, so a warp
//                 keeps several columns of HBM traffic outstanding.
//   kVariantLdg   plain 128-bit read-only loads into registers.
//
// Traffic per cell-update: px, pz, vx, vz read once and written once
// (32 B) and kappa, bx, bz read once (12 B, shared through L2 by the shots
// of a batch that use the same model).  Where both pressure dampings are 1
// (the model's interior) the cell carries p = px + pz alone and pz is neither
// read nor written: 36 B.
#include <cuda_runtime.h>
#include <cstdint>

#include "s2d_device.cuh"

namespace s2d {

namespace {

// The two arithmetic forms of the update, with the rounding of every
// operation fixed (explicit fma/mul, nothing left to contraction), so that a
// row computes the same bits whether its coefficients are literals or loads.
//   dif: c0*d0 + c1*d1, one product rounded, then fused;
//   upd: a*x + (b*k)*d, the coefficient product and the term rounded, then fused.
__device__ __forceinline__ float dif(float c0, float d0, float c1, float d1) {
    return __fmaf_rn(c0, d0, __fmul_rn(c1, d1));
}
__device__ __forceinline__ float upd(float a, float x, float b, float k, float d) {
    return __fmaf_rn(a, x, __fmul_rn(__fmul_rn(b, k), d));
}

// One cell of the pressure update.  Split (the reference's form): px and pz
// damped separately.  Merged (both pressure dampings exactly 1): px and pz
// only enter through p = px + pz, so the cell carries p in px (pz stays 0):
//   p' = p + kappa (Kx Dx vx + Kz Dz vz).
// The product saved for the gradient is Dx vx (split) or Kx Dx vx + Kz Dz vz
// (merged) in the first slot, Dz vz (split) or 0 in the second.
__device__ __forceinline__ void p_cell(bool merged, float dax, float kx, float daz, float kz, float px, float pz,
                                       float k, float dx, float dz, float &pxn, float &pzn, float &t0, float &t1) {
    if (merged) {
        const float t = dif(kx, dx, kz, dz);
        pxn = __fmaf_rn(k, t, px);
        pzn = 0.0f;
        t0 = t;
        t1 = 0.0f;
    } else {
        pxn = upd(dax, px, kx, k, dx);
        pzn = upd(daz, pz, kz, k, dz);
        t0 = dx;
        t1 = dz;
    }
}

// Pressure at column P from vx at P-2..P+1 (q0..q3), old px, pz, kappa and vz
// at P (cpu_modelling_kernels.cpp:201-258 and 335-351, cpumodelling.cpp:136-142).
// xc = (Dax, Kx, Dbx, Lx) of column P; colm: Dax == 1 (FAST tasks then have
// every cell merged and pz is not read).  Returns new p; new px, pz in pxn,
// pzn; the step's products in dxv, dzv.
// XF: column P lies in the shot's x-interior (operator pair (a0, a1)).
template <bool FAST, bool XF = false>
__device__ __forceinline__ float4 p_update(const Lane<FAST> &ln, const ShotDev &S, int P, const float4 &xc,
                                           bool colm, const float4 &q0, const float4 &q1, const float4 &q2,
                                           const float4 &q3, const float4 &px, const float4 &pz, const float4 &kk,
                                           const float4 &vz, float4 &pxn, float4 &pzn, float4 &dxv, float4 &dzv) {
    float cx0 = kA0, cx1 = kA1;
    if (!XF) dm_coef(P, S.nnx, cx0, cx1);
    const float up_z = __shfl_up_sync(kFull, vz.z, 1);
    const float up_w = __shfl_up_sync(kFull, vz.w, 1);
    const float dn_x = __shfl_down_sync(kFull, vz.x, 1);
    float a0, a1;
    zdm(ln, 0, a0, a1);
    const float dz0 = dif(a0, vz.x - up_w, a1, vz.y - up_z);
    zdm(ln, 1, a0, a1);
    const float dz1 = dif(a0, vz.y - vz.x, a1, vz.z - up_w);
    zdm(ln, 2, a0, a1);
    const float dz2 = dif(a0, vz.z - vz.y, a1, vz.w - vz.x);
    zdm(ln, 3, a0, a1);
    const float dz3 = dif(a0, vz.w - vz.z, a1, dn_x - vz.y);
    const float dx0 = dif(cx0, q2.x - q1.x, cx1, q3.x - q0.x);
    const float dx1 = dif(cx0, q2.y - q1.y, cx1, q3.y - q0.y);
    const float dx2 = dif(cx0, q2.z - q1.z, cx1, q3.z - q0.z);
    const float dx3 = dif(cx0, q2.w - q1.w, cx1, q3.w - q0.w);
    // z-damping of the lane's rows (FAST: 1, the cell is merged iff colm)
    const float4 r0 = zrow(ln, 0), r1 = zrow(ln, 1), r2 = zrow(ln, 2), r3 = zrow(ln, 3);
    p_cell(colm && (FAST || r0.x == 1.0f), xc.x, xc.y, r0.x, r0.y, px.x, pz.x, kk.x, dx0, dz0, pxn.x, pzn.x, dxv.x,
           dzv.x);
    p_cell(colm && (FAST || r1.x == 1.0f), xc.x, xc.y, r1.x, r1.y, px.y, pz.y, kk.y, dx1, dz1, pxn.y, pzn.y, dxv.y,
           dzv.y);
    p_cell(colm && (FAST || r2.x == 1.0f), xc.x, xc.y, r2.x, r2.y, px.z, pz.z, kk.z, dx2, dz2, pxn.z, pzn.z, dxv.z,
           dzv.z);
    p_cell(colm && (FAST || r3.x == 1.0f), xc.x, xc.y, r3.x, r3.y, px.w, pz.w, kk.w, dx3, dz3, pxn.w, pzn.w, dxv.w,
           dzv.w);
    if (P == ln.src_x && ln.sdz >= 0 && ln.sdz < 4) {
        if (ln.sdz == 0) pxn.x += ln.amp;
        else if (ln.sdz == 1) pxn.y += ln.amp;
        else if (ln.sdz == 2) pxn.z += ln.amp;
        else pxn.w += ln.amp;
    }
    // merged cells: pzn = 0 and p = px exactly
    return make_float4(pxn.x + pzn.x, pxn.y + pzn.y, pxn.z + pzn.z, pxn.w + pzn.w);
}

// Receiver sampling of new p at column P (cpumodelling.cpp:356-360).
template <bool FAST>
__device__ __forceinline__ void record(const Lane<FAST> &ln, const ShotDev &S, int P, const float4 &pn, int slot) {
    const int j1 = __ldg(S.rec_ptr + P + 1);
    for (int j = __ldg(S.rec_ptr + P); j < j1; ++j) {
        const int d = __ldg(S.rec_z + j) - ln.z0;
        if (ln.owner && d >= 0 && d < 4) S.seis[(size_t)__ldg(S.rec_id + j) * S.real_nt + slot] = comp(pn, d);
    }
}

// Velocities at column V from new p at V-1..V+2 (p0..p3), old vx, vz at V and
// bx, bz at V (cpu_modelling_kernels.cpp:260-316 and 353-368); D+x p and D+z p
// in dxp, dzp.
// XF: column V lies in the shot's x-interior: x-dampings 1, Lx = kx_in,
// operator pair (a0, a1), no coefficient load.
template <bool FAST, bool XF = false>
__device__ __forceinline__ void v_update(const Lane<FAST> &ln, const ShotDev &S, int V, const float4 &p0,
                                         const float4 &p1, const float4 &p2, const float4 &p3, const float4 &vx,
                                         const float4 &vz, const float4 &bx, const float4 &bz, float4 &vxn,
                                         float4 &vzn, float4 &dxp, float4 &dzp) {
    const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (V + S2D_GX));
    float ux0 = kA0, ux1 = kA1;
    if (!XF) dp_coef(V, S.nnx, ux0, ux1);
    const float ex0 = dif(ux0, p2.x - p1.x, ux1, p3.x - p0.x);
    const float ex1 = dif(ux0, p2.y - p1.y, ux1, p3.y - p0.y);
    const float ex2 = dif(ux0, p2.z - p1.z, ux1, p3.z - p0.z);
    const float ex3 = dif(ux0, p2.w - p1.w, ux1, p3.w - p0.w);
    const float4 q = p1;
    const float up_w = __shfl_up_sync(kFull, q.w, 1);
    const float dn_x = __shfl_down_sync(kFull, q.x, 1);
    const float dn_y = __shfl_down_sync(kFull, q.y, 1);
    float b0, b1;
    zdp(ln, 0, b0, b1);
    const float ez0 = dif(b0, q.y - q.x, b1, q.z - up_w);
    zdp(ln, 1, b0, b1);
    const float ez1 = dif(b0, q.z - q.y, b1, q.w - q.x);
    zdp(ln, 2, b0, b1);
    const float ez2 = dif(b0, q.w - q.z, b1, dn_x - q.y);
    zdp(ln, 3, b0, b1);
    const float ez3 = dif(b0, dn_x - q.w, b1, dn_y - q.z);
    dxp = make_float4(ex0, ex1, ex2, ex3);
    dzp = make_float4(ez0, ez1, ez2, ez3);
    vxn.x = upd(xc.z, vx.x, xc.w, bx.x, ex0);
    vxn.y = upd(xc.z, vx.y, xc.w, bx.y, ex1);
    vxn.z = upd(xc.z, vx.z, xc.w, bx.z, ex2);
    vxn.w = upd(xc.z, vx.w, xc.w, bx.w, ex3);
    float4 r = zrow(ln, 0);
    vzn.x = upd(r.z, vz.x, r.w, bz.x, ez0);
    r = zrow(ln, 1);
    vzn.y = upd(r.z, vz.y, r.w, bz.y, ez1);
    r = zrow(ln, 2);
    vzn.z = upd(r.z, vz.z, r.w, bz.z, ez2);
    r = zrow(ln, 3);
    vzn.w = upd(r.z, vz.w, r.w, bz.w, ez3);
}

// ---------------------------------------------------------------- LDG variant

// Per-task constants of the plain-load loop.
template <bool PROD, bool FAST>
struct LdgTask {
    Lane<FAST> ln;
    int xa, xb, slot;
    bool rec;
    ptrdiff_t ld;
    size_t F;
    const float *__restrict__ pxi;
    const float *__restrict__ pzi;
    const float *__restrict__ vxi;
    const float *__restrict__ vzi;
    float *__restrict__ pxo;
    float *__restrict__ pzo;
    float *__restrict__ vxo;
    float *__restrict__ vzo;
    const float *__restrict__ kap;
    const float *__restrict__ bxp;
    const float *__restrict__ bzp;
    float *__restrict__ pr;
};

// The loads of one column L: vx(L); px, pz, kappa, vz at L-1; bx, bz at L-3.
struct ColIn {
    float4 vx, px, pz, k, vz, bx, bz;
};
// State loads: the read-only path, or (CG) loads cached in L2 only, for a
// kernel that reads in one step what another block wrote in the previous
// step of the same launch.
template <bool CG>
__device__ __forceinline__ float4 ld4s(const float *p) {
    if (CG) return __ldcg(reinterpret_cast<const float4 *>(p));
    return __ldg(reinterpret_cast<const float4 *>(p));
}

template <bool PROD, bool FAST, bool XF, bool CG = false>
__device__ __forceinline__ void ldg_load(const LdgTask<PROD, FAST> &k, const ShotDev &S, int L, ColIn &in) {
    const ptrdiff_t colL = (ptrdiff_t)L * k.ld, colP = colL - k.ld, colV = colL - 3 * k.ld;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    in.vx = ld4s<CG>(k.vxi + colL);
    in.px = ld4s<CG>(k.pxi + colP);
    const bool pz_live = !(FAST && (XF || __ldg(S.xcoef + (L - 1 + S2D_GX)).x == 1.0f));
    in.pz = pz_live ? ld4s<CG>(k.pzi + colP) : zero;
    in.k = ld4(k.kap + colP);
    in.vz = ld4s<CG>(k.vzi + colP);
    in.bx = ld4(k.bxp + colV);
    in.bz = ld4(k.bzp + colV);
}

// One column L of the loop from its loaded inputs (the prefetching form of
// ldg_column below; same arithmetic).
template <bool PROD, bool FAST, bool XF>
__device__ __forceinline__ void ldg_column_in(const LdgTask<PROD, FAST> &k, const ShotDev &S, int L,
                                              const ColIn &in, float4 &vo, const float4 &v1, const float4 &v2,
                                              const float4 &v3, float4 &po, const float4 &p1, const float4 &p2,
                                              const float4 &p3, float4 &zo, const float4 &z2) {
    const int P = L - 1;
    const ptrdiff_t colP = (ptrdiff_t)P * k.ld;
    vo = in.vx;
    const float4 xc = XF ? make_float4(1.0f, k.ln.kx, 1.0f, k.ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
    const bool colm = XF || xc.x == 1.0f;
    const bool pz_live = !(FAST && colm);
    float4 pxn, pzn, dxv, dzv;
    const float4 pn = p_update<FAST, XF>(k.ln, S, P, xc, colm, v1, v2, v3, vo, in.px, in.pz, in.k, in.vz, pxn, pzn,
                                         dxv, dzv);
    const bool in_seg = P >= k.xa && P < k.xb;
    if (in_seg && k.ln.owner) {
        st4(k.pxo + colP, pxn);
        if (pz_live) st4(k.pzo + colP, pzn);
        if (PROD) {
            st4(k.pr + colP, dxv);
            if (pz_live) st4(k.pr + k.F + colP, dzv);
        }
    }
    if (k.rec && in_seg) record(k.ln, S, P, pn, k.slot);
    po = pn;
    zo = in.vz;
    if (L >= k.xa + 3) {
        const int V = L - 3;
        const ptrdiff_t colV = (ptrdiff_t)V * k.ld;
        float4 vxn, vzn, dxp, dzp;
        v_update<FAST, XF>(k.ln, S, V, p1, p2, p3, po, v1, z2, in.bx, in.bz, vxn, vzn, dxp, dzp);
        if (k.ln.owner) {
            st4(k.vxo + colV, vxn);
            st4(k.vzo + colV, vzn);
            if (PROD) {
                st4(k.pr + 2 * k.F + colV, dxp);
                st4(k.pr + 3 * k.F + colV, dzp);
            }
        }
    }
}

// One column L of the loop: vx(L) into vo (the window vx(L-3 .. L) is then
// v1, v2, v3, vo), new p at P = L-1 into po (p(P-3 .. P) is p1, p2, p3, po),
// vz(P) into zo (z2 holds vz(P-2)), velocities at V = L-3.  The caller
// passes the window registers in rotated order, so the windows slide without
// moves.  XF: every column of the task lies in the shot's x-interior.
template <bool PROD, bool FAST, bool XF>
__device__ __forceinline__ void ldg_column(const LdgTask<PROD, FAST> &k, const ShotDev &S, int L, float4 &vo,
                                           const float4 &v1, const float4 &v2, const float4 &v3, float4 &po,
                                           const float4 &p1, const float4 &p2, const float4 &p3, float4 &zo,
                                           const float4 &z2) {
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const int P = L - 1;
    const ptrdiff_t colP = (ptrdiff_t)P * k.ld;
    vo = ld4(k.vxi + (ptrdiff_t)L * k.ld);
    const float4 vz = ld4(k.vzi + colP);
    const float4 xc = XF ? make_float4(1.0f, k.ln.kx, 1.0f, k.ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
    const bool colm = XF || xc.x == 1.0f;
    const bool pz_live = !(FAST && colm);  // some cell of the column keeps pz
    float4 pxn, pzn, dxv, dzv;
    const float4 pn = p_update<FAST, XF>(k.ln, S, P, xc, colm, v1, v2, v3, vo, ld4(k.pxi + colP),
                                         pz_live ? ld4(k.pzi + colP) : zero, ld4(k.kap + colP), vz, pxn, pzn, dxv,
                                         dzv);
    const bool in_seg = P >= k.xa && P < k.xb;
    if (in_seg && k.ln.owner) {
        st4(k.pxo + colP, pxn);
        if (pz_live) st4(k.pzo + colP, pzn);
        if (PROD) {
            st4(k.pr + colP, dxv);
            if (pz_live) st4(k.pr + k.F + colP, dzv);
        }
    }
    if (k.rec && in_seg) record(k.ln, S, P, pn, k.slot);
    po = pn;
    zo = vz;
    if (L >= k.xa + 3) {
        const int V = L - 3;
        const ptrdiff_t colV = (ptrdiff_t)V * k.ld;
        float4 vxn, vzn, dxp, dzp;
        v_update<FAST, XF>(k.ln, S, V, p1, p2, p3, po, v1, z2, ld4(k.bxp + colV), ld4(k.bzp + colV), vxn, vzn,
                           dxp, dzp);
        if (k.ln.owner) {
            st4(k.vxo + colV, vxn);
            st4(k.vzo + colV, vzn);
            if (PROD) {
                st4(k.pr + 2 * k.F + colV, dxp);
                st4(k.pr + 3 * k.F + colV, dzp);
            }
        }
    }
}

// One (shot, strip, segment) task of the plain-load kernel.  PROD: also write
// the step's four derivatives (gradient runs, S2D_STEP_PRODUCTS).  U4: the
// column loop unrolled by 4 with the windows rotating through the register
// names (no moves); otherwise one column per iteration.  PF: the loads of
// column L+1 are issued before column L is computed (two columns of loads in
// flight per warp).
template <bool PROD, bool FAST, bool XF, bool U4, bool PF = false, bool CG = false>
__device__ __forceinline__ void ldg_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len,
                                         int kt, int par, bool rec_step, int slot, int lane) {
    LdgTask<PROD, FAST> k;
    k.xa = xa;
    k.xb = min(S.nnx, xa + seg_len);
    k.ld = (ptrdiff_t)S.ld;
    const int c = strip * S2D_STRIP_OUT - 4;
    lane_setup(k.ln, S, c, lane, kt);
    // receivers only where the strip's rows hold some
    k.rec = rec_step && slot < S.real_nt && !(a.flags & S2D_STEP_NO_RECORD) && c + S2D_STRIP_ROWS > S.rec_zlo &&
            c <= S.rec_zhi;
    k.slot = slot;
    const size_t off = (size_t)(k.ln.zl + S2D_GZ) + (size_t)S2D_GX * (size_t)S.ld;
    k.F = (size_t)(S.nnx + 2 * S2D_GX) * (size_t)S.ld;
    k.pr = PROD ? S.prod + (size_t)(kt - a.prod_kt0) * 4 * k.F + off : nullptr;
    // every field from one base and a 32-bit stride (fewer live registers
    // than eleven 64-bit pointers)
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off;
    const int ib = par * 4 * fs, ob = (par ^ 1) * 4 * fs;
    k.pxi = sb + ib;
    k.pzi = sb + ib + fs;
    k.vxi = sb + ib + 2 * fs;
    k.vzi = sb + ib + 3 * fs;
    k.pxo = sb + ob;
    k.pzo = sb + ob + fs;
    k.vxo = sb + ob + 2 * fs;
    k.vzo = sb + ob + 3 * fs;
    k.kap = S.kappa + off;
    k.bxp = k.kap + fs;
    k.bzp = k.kap + 2 * fs;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    // windows: vx(L-4 .. L-1), p(P-4 .. P-1), vz(P-4 .. P-1) before column L
    float4 vA = zero, vB, vC, vD;
    float4 pA = zero, pB = zero, pC = zero, pD = zero;
    float4 zA = zero, zB = zero, zC = zero, zD = zero;
    vB = ld4s<CG>(k.vxi + (ptrdiff_t)(xa - 3) * k.ld);
    vC = ld4s<CG>(k.vxi + (ptrdiff_t)(xa - 2) * k.ld);
    vD = ld4s<CG>(k.vxi + (ptrdiff_t)(xa - 1) * k.ld);
    const int Lend = k.xb + 2;
    int L = xa;
    if (PF && U4) {
        // two load buffers in turn and the windows rotating through the
        // register names: no moves in the unrolled body
        ColIn X, Y;
        ldg_load<PROD, FAST, XF>(k, S, L, X);
        for (; L + 3 <= Lend; L += 4) {
            ldg_load<PROD, FAST, XF>(k, S, L + 1, Y);
            ldg_column_in<PROD, FAST, XF>(k, S, L, X, vA, vB, vC, vD, pA, pB, pC, pD, zA, zC);
            ldg_load<PROD, FAST, XF>(k, S, L + 2, X);
            ldg_column_in<PROD, FAST, XF>(k, S, L + 1, Y, vB, vC, vD, vA, pB, pC, pD, pA, zB, zD);
            ldg_load<PROD, FAST, XF>(k, S, L + 3, Y);
            ldg_column_in<PROD, FAST, XF>(k, S, L + 2, X, vC, vD, vA, vB, pC, pD, pA, pB, zC, zA);
            if (L + 4 <= Lend) ldg_load<PROD, FAST, XF>(k, S, L + 4, X);
            ldg_column_in<PROD, FAST, XF>(k, S, L + 3, Y, vD, vA, vB, vC, pD, pA, pB, pC, zD, zB);
        }
        // X holds column L's loads
        for (; L <= Lend; ++L) {
            const ColIn cur = X;
            if (L < Lend) ldg_load<PROD, FAST, XF>(k, S, L + 1, X);
            ldg_column_in<PROD, FAST, XF>(k, S, L, cur, vA, vB, vC, vD, pA, pB, pC, pD, zA, zC);
            float4 t = vA;
            vA = vB; vB = vC; vC = vD; vD = t;
            t = pA;
            pA = pB; pB = pC; pC = pD; pD = t;
            t = zA;
            zA = zB; zB = zC; zC = zD; zD = t;
        }
        return;
    }
    if (PF) {
        ColIn cur, nxt;
        ldg_load<PROD, FAST, XF, CG>(k, S, L, nxt);
        for (; L <= Lend; ++L) {
            cur = nxt;
            if (L < Lend) ldg_load<PROD, FAST, XF, CG>(k, S, L + 1, nxt);
            ldg_column_in<PROD, FAST, XF>(k, S, L, cur, vA, vB, vC, vD, pA, pB, pC, pD, zA, zC);
            float4 t = vA;
            vA = vB; vB = vC; vC = vD; vD = t;
            t = pA;
            pA = pB; pB = pC; pC = pD; pD = t;
            t = zA;
            zA = zB; zB = zC; zC = zD; zD = t;
        }
        return;
    }
    if (U4) {
        for (; L + 3 <= Lend; L += 4) {
            ldg_column<PROD, FAST, XF>(k, S, L, vA, vB, vC, vD, pA, pB, pC, pD, zA, zC);
            ldg_column<PROD, FAST, XF>(k, S, L + 1, vB, vC, vD, vA, pB, pC, pD, pA, zB, zD);
            ldg_column<PROD, FAST, XF>(k, S, L + 2, vC, vD, vA, vB, pC, pD, pA, pB, zC, zA);
            ldg_column<PROD, FAST, XF>(k, S, L + 3, vD, vA, vB, vC, pD, pA, pB, pC, zD, zB);
        }
    }
    for (; L <= Lend; ++L) {
        ldg_column<PROD, FAST, XF>(k, S, L, vA, vB, vC, vD, pA, pB, pC, pD, zA, zC);
        float4 t = vA;
        vA = vB; vB = vC; vC = vD; vD = t;
        t = pA;
        pA = pB; pB = pC; pC = pD; pD = t;
        t = zA;
        zA = zB; zB = zC; zC = zD; zD = t;
    }
}

// MINB = 4 caps registers at 128 (4 blocks of 4 warps per SM, some spill);
// MINB = 3 keeps the product-writing instance at 3 blocks per SM.
template <bool PROD, int MINB, bool U4 = false, bool PF = false>
__global__ void __launch_bounds__(128, MINB) step_kernel_ldg(const StepArgs *__restrict__ A, int kt_off) {
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    const int par = a.par0 ^ (kt_off & 1);
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        if (!task_in_bounds(a, G, strip, xa, seg_len, kt, PROD, 1)) continue;
        warp_copy_shot(S, G, lane);
        const int c = strip * S2D_STRIP_OUT - 4;
        const int xb = min(S.nnx, xa + seg_len);
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
        // columns xa-1 .. xb+1 take part (p there, v on xa .. xb-1)
        const bool xf = xa - 1 >= S.xfast_lo && xb + 1 < S.xfast_hi;
        if (zf && xf) ldg_task<PROD, true, true, U4, PF>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else if (zf) ldg_task<PROD, true, false, U4, PF>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else if (xf) ldg_task<PROD, false, true, U4, PF>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else ldg_task<PROD, false, false, U4, PF>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
    }
}

// ---------------------------------------------------------- persistent variant
//
// One launch advances up to `nsteps` FD steps: every warp runs its tasks of
// a step (the prefetching plain-load loop), then the grid meets at a barrier
// before the next step, so a run of small grids (one shot, one round of
// tasks per step) pays one launch per chunk of steps instead of one per
// step.  The grid is exactly the co-resident blocks (a cooperative launch).
// State written in step k is read by other blocks in step k+1 of the same
// launch, so state loads take the L2-only path (ld.global.cg) and each block
// fences its stores before it arrives.  The barrier is a counter that every
// block increments once per step; a block waits (bounded: spin_limit polls)
// for (k+1) x gridDim.x arrivals.  A wait that runs out records
// S2D_DEV_ERR_WAIT and the block leaves; the call then returns
// S2D_ERR_TIMEOUT.  Test knob fault_iter: block 0 does not arrive after step
// fault_iter, so every wait of that step runs out.

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) step_kernel_persist(const StepArgs *__restrict__ A, int nsteps,
                                                                  unsigned *bar) {
    __shared__ int s_ok;
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    for (int s = 0; s < nsteps; ++s) {
        const int kt = a.kt_base + s;
        if (kt >= a.fd_nt) return;
        const int par = a.par0 ^ (s & 1);
        const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
        const int slot = (kt + 1) / a.dt_factor - 1;
        for (int t = gwarp; t < a.total_tasks; t += nwarp) {
            int strip, xa, seg_len;
            const ShotDev &S = task_of(a, t, strip, xa, seg_len);
            if (!task_in_bounds(a, S, strip, xa, seg_len, kt, false, 1)) continue;
            const int c = strip * S2D_STRIP_OUT - 4;
            const int xb = min(S.nnx, xa + seg_len);
            const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
            const bool xf = xa - 1 >= S.xfast_lo && xb + 1 < S.xfast_hi;
            if (zf && xf)
                ldg_task<false, true, true, false, true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
            else if (zf)
                ldg_task<false, true, false, false, true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
            else if (xf)
                ldg_task<false, false, true, false, true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
            else
                ldg_task<false, false, false, false, true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot,
                                                                 lane);
        }
        if (s + 1 == nsteps) break;
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (!(s == a.fault_iter && blockIdx.x == 0)) atomicAdd(bar, 1u);
            const unsigned target = (unsigned)(s + 1) * gridDim.x;
            bool ok = false;
            for (int i = 0; i < a.spin_limit && !ok; ++i) {
                ok = ld_acquire_gpu(bar) >= target;
                if (!ok) __nanosleep(64);
            }
            if (!ok) atomicOr(a.err, S2D_DEV_ERR_WAIT);
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return;
    }
}

// --------------------------------------------------------------- bulk variant

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bounded wait: every lane polls; the warp agrees on the outcome.
__device__ __forceinline__ bool wait_stage(uint64_t *bar, unsigned parity, int limit) {
    bool ok = false;
    for (int i = 0; i < limit && !ok; ++i) ok = mbar_try_wait(bar, parity);
    return __all_sync(kFull, ok);
}

constexpr int kDrainLimit = 1 << 20;

// One task of the bulk-copy kernel; returns false when a pipeline wait gave up
// (the warp must then leave the kernel).
template <bool FAST>
__device__ __forceinline__ bool bulk_task(const StepArgs &a, const ShotDev &Sh, int strip, int xa, int seg_len,
                                          int kt, int par, bool rec_step, int slot, int lane, unsigned char *ring,
                                          uint64_t *bars, int S, int drain_limit, unsigned &it0) {
    const int xb = min(Sh.nnx, xa + seg_len);
    const size_t ld = (size_t)Sh.ld;
    const int c = strip * S2D_STRIP_OUT - 4;
    Lane<FAST> ln;
    lane_setup(ln, Sh, c, lane, kt);
    const bool rec = rec_step && slot < Sh.real_nt && !(a.flags & S2D_STEP_NO_RECORD);
    // column 0 of the warp's strip in each field (row c), and this lane's rows
    const size_t wofs = (size_t)(c + S2D_GZ) + (size_t)S2D_GX * ld;
    const size_t lofs = wofs + (size_t)(S2D_ZPT * lane);
    const int fs = Sh.fstride;
    const float *src_px = Sh.st[0][0] + wofs + par * 4 * fs;
    const float *src_pz = src_px + fs, *src_vx = src_px + 2 * fs, *src_vz = src_px + 3 * fs;
    const float *src_k = Sh.kappa + wofs, *src_bx = src_k + fs, *src_bz = src_k + 2 * fs;
    float *pxo = Sh.st[0][0] + lofs + (par ^ 1) * 4 * fs, *pzo = pxo + fs;
    float *vxo = pxo + 2 * fs, *vzo = pxo + 3 * fs;
    const int n_it = xb - xa + 6;  // columns L = xa-3 .. xb+2

    // Producer (lane 0): bring iteration j's columns into stage (it0+j) % S.
    auto issue = [&](int j) {
        const unsigned itj = it0 + (unsigned)j;
        const int s = (int)(itj % (unsigned)S);
        unsigned char *st = ring + (size_t)s * kStageBytes;
        const int L = xa - 3 + j;
        const bool pp = L >= xa, vv = L >= xa + 3;
        // pz of column L-1 is not needed where every cell is merged
        const bool pz = pp && !(FAST && __ldg(Sh.xcoef + (L - 1 + S2D_GX)).x == 1.0f);
        mbar_expect_tx(&bars[s], (unsigned)kSlotBytes * (1u + (pp ? 3u : 0u) + (pz ? 1u : 0u) + (vv ? 2u : 0u)));
        if (j == a.fault_iter) return;  // test knob: the stage's bytes never arrive
        bulk_copy(st, src_vx + (ptrdiff_t)L * (ptrdiff_t)ld, kSlotBytes, &bars[s]);
        if (pp) {
            const ptrdiff_t cp = (ptrdiff_t)(L - 1) * (ptrdiff_t)ld;
            bulk_copy(st + 1 * kSlotBytes, src_px + cp, kSlotBytes, &bars[s]);
            if (pz) bulk_copy(st + 2 * kSlotBytes, src_pz + cp, kSlotBytes, &bars[s]);
            bulk_copy(st + 3 * kSlotBytes, src_k + cp, kSlotBytes, &bars[s]);
            bulk_copy(st + 4 * kSlotBytes, src_vz + cp, kSlotBytes, &bars[s]);
        }
        if (vv) {
            const ptrdiff_t cv = (ptrdiff_t)(L - 3) * (ptrdiff_t)ld;
            bulk_copy(st + 5 * kSlotBytes, src_bx + cv, kSlotBytes, &bars[s]);
            bulk_copy(st + 6 * kSlotBytes, src_bz + cv, kSlotBytes, &bars[s]);
        }
    };
    if (lane == 0) {
        const int pre = min(S, n_it);
        for (int j = 0; j < pre; ++j) issue(j);
    }

    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 vq0 = zero, vq1 = zero, vq2 = zero, vq3 = zero;
    float4 pq0 = zero, pq1 = zero, pq2 = zero, pq3 = zero;
    float4 zq0 = zero, zq1 = zero, zq2 = zero;
    for (int j = 0; j < n_it; ++j) {
        const unsigned itj = it0 + (unsigned)j;
        const int s = (int)(itj % (unsigned)S);
        if (!wait_stage(&bars[s], (itj / (unsigned)S) & 1u, a.spin_limit)) {
            // Give up: record the error, let the copies already issued
            // land (bounded), and leave without touching global state.
            if (lane == 0) atomicOr(a.err, S2D_DEV_ERR_WAIT);
            const int last = min(n_it, j + S);
            for (int k = j; k < last; ++k) {
                const unsigned itk = it0 + (unsigned)k;
                if (!wait_stage(&bars[itk % (unsigned)S], (itk / (unsigned)S) & 1u, drain_limit)) {
                    if (lane == 0) atomicOr(a.err, S2D_DEV_ERR_DRAIN);
                }
            }
            return false;
        }
        const float4 *st = reinterpret_cast<const float4 *>(ring + (size_t)s * kStageBytes) + lane;
        const int L = xa - 3 + j;
        vq0 = vq1; vq1 = vq2; vq2 = vq3;
        vq3 = st[0 * 32];
        if (L >= xa) {
            const int P = L - 1;
            const float4 vz = st[4 * 32];
            const float4 xc = __ldg(Sh.xcoef + (P + S2D_GX));
            const bool colm = xc.x == 1.0f;
            const bool pz_live = !(FAST && colm);
            float4 pxn, pzn, dxv, dzv;
            const float4 pn = p_update(ln, Sh, P, xc, colm, vq0, vq1, vq2, vq3, st[1 * 32],
                                       pz_live ? st[2 * 32] : zero, st[3 * 32], vz, pxn, pzn, dxv, dzv);
            const bool in_seg = P >= xa && P < xb;
            const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
            if (in_seg && ln.owner) {
                st4(pxo + colP, pxn);
                if (pz_live) st4(pzo + colP, pzn);
            }
            if (rec && in_seg) record(ln, Sh, P, pn, slot);
            pq0 = pq1; pq1 = pq2; pq2 = pq3; pq3 = pn;
            zq0 = zq1; zq1 = zq2; zq2 = vz;
            if (L >= xa + 3) {
                const int V = L - 3;
                const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
                float4 vxn, vzn, dxp, dzp;
                v_update(ln, Sh, V, pq0, pq1, pq2, pq3, vq0, zq0, st[5 * 32], st[6 * 32], vxn, vzn, dxp, dzp);
                if (ln.owner) {
                    st4(vxo + colV, vxn);
                    st4(vzo + colV, vzn);
                }
            }
        }
        __syncwarp();
        if (lane == 0 && j + S < n_it) {
            fence_proxy_async();
            issue(j + S);
        }
    }
    it0 += (unsigned)n_it;
    return true;
}

// MINB = 1 lets the compiler use the registers it wants, MINB = 4 caps it at
// 128 (4 blocks per SM).
template <int MINB>
__global__ void __launch_bounds__(128, MINB) step_kernel_bulk(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    // an earlier launch of this sequence gave up: its wavefields are not valid
    if (*reinterpret_cast<volatile int *>(a.err) != 0) return;
    const int S = a.stages;
    const int drain_limit = a.spin_limit < kDrainLimit / 64 ? a.spin_limit * 64 : kDrainLimit;
    unsigned char *ring = smem + (size_t)wib * S * kStageBytes;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)wpb * S * kStageBytes) + wib * S;
    if (lane == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
    }
    __syncwarp();
    const int par = a.par0 ^ (kt_off & 1);
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    unsigned it0 = 0;  // pipeline iterations consumed by this warp so far
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &Sh = task_of(a, t, strip, xa, seg_len);
        const int c = strip * S2D_STRIP_OUT - 4;
        const bool ok = rows_fast(Sh, c, c + S2D_STRIP_ROWS - 1)
                            ? bulk_task<true>(a, Sh, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring, bars,
                                              S, drain_limit, it0)
                            : bulk_task<false>(a, Sh, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring, bars,
                                               S, drain_limit, it0);
        if (!ok) return;
    }
}

// ------------------------------------------------------------ two-step variant
//
// One launch advances the batch by two FD steps (kt, kt+1): the state is read
// from HBM once and written once per two steps.  The warp streams along x as
// the one-step kernel does; step A (kt) runs at the front of the stream and
// step B (kt+1) trails it:
//   column L of vx (step-A input) is loaded at loop index L;
//   step A: p at L-1, v at L-3 (as in the one-step kernel);
//   step B: p at L-4 (needs step-A vx at L-6 .. L-3), v at L-6 (needs step-B p
//           at L-7 .. L-4).
// Step-A results never reach HBM: px, pz, vz and vx of step A and the
// step-B pressure wait in per-warp shared-memory delay lines of 4 columns
// (each lane reads back only what it wrote), which also serve as step B's
// x-stencil windows, so the kernel fits 128 registers (4 blocks per SM);
// kappa, bx, bz are read again for step B (L1/L2 hits: DRAM reads them once).  Two steps of z-halo leave lanes 2..29 valid
// (rows c+8 .. c+119 of a strip starting at c = 112k - 8), so strips write
// 112 rows; the segment's stream starts 6 columns early and ends 5 late.
// TWO = false is the same kernel doing step A alone (odd remainders), in the
// same strip layout.

__device__ __forceinline__ float4 &ring_at(float4 *ring, int field, int col, int lane) {
    return ring[(field * kTsRing + ((col + 2 * S2D_GX) & (kTsRing - 1))) * 32 + lane];
}

// XF: every column either step updates or differentiates (xa-4 .. xb+4)
// lies in the shot's x-interior: literal column coefficients.
template <bool FAST, bool TWO, bool XF = false>
__device__ __forceinline__ void ts_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len,
                                        int kt, int par, int lane, float4 *ring) {
    const int xb = min(S.nnx, xa + seg_len);
    const size_t ld = (size_t)S.ld;
    const int c = strip * S2D_TS_OUT - 8;
    Lane<FAST> la;
    lane_setup(la, S, c, lane, kt);
    la.owner = lane >= 2 && lane <= 29;
    Lane<FAST> lb = la;
    if (TWO) lb.amp = __ldg(S.amp + kt + 1);
    const bool rec = !(a.flags & S2D_STEP_NO_RECORD);
    const bool rec_a = rec && ((kt + 1) % a.dt_factor) == 0 && (kt + 1) / a.dt_factor - 1 < S.real_nt;
    const int slot_a = (kt + 1) / a.dt_factor - 1;
    const bool rec_b = TWO && rec && ((kt + 2) % a.dt_factor) == 0 && (kt + 2) / a.dt_factor - 1 < S.real_nt;
    const int slot_b = (kt + 2) / a.dt_factor - 1;
    const size_t off = (size_t)(la.z0 + S2D_GZ) + (size_t)S2D_GX * ld;
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off;
    const int ib = par * 4 * fs, ob = (par ^ 1) * 4 * fs;
    const float *__restrict__ pxi = sb + ib;
    const float *__restrict__ pzi = sb + ib + fs;
    const float *__restrict__ vxi = sb + ib + 2 * fs;
    const float *__restrict__ vzi = sb + ib + 3 * fs;
    float *__restrict__ pxo = sb + ob;
    float *__restrict__ pzo = sb + ob + fs;
    float *__restrict__ vxo = sb + ob + 2 * fs;
    float *__restrict__ vzo = sb + ob + 3 * fs;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = kap + fs;
    const float *__restrict__ bzp = kap + 2 * fs;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    // step A windows: vx at L-3..L, new p at L-4..L-1, vz at L-3..L-1
    float4 vq0 = zero, vq1, vq2, vq3;
    float4 pq0 = zero, pq1 = zero, pq2 = zero, pq3 = zero;
    float4 zq0 = zero, zq1 = zero, zq2 = zero;
    // step B windows: step-A vx at L-6..L-3, step-B p at L-7..L-4
    const int h = TWO ? 3 : 0;  // step A runs over [xa - h, xb + h)
    const int xaa = xa - h, xba = xb + h;
    vq1 = ld4(vxi + (ptrdiff_t)(xaa - 3) * (ptrdiff_t)ld);
    vq2 = ld4(vxi + (ptrdiff_t)(xaa - 2) * (ptrdiff_t)ld);
    vq3 = ld4(vxi + (ptrdiff_t)(xaa - 1) * (ptrdiff_t)ld);
    for (int L = xaa; L <= xba + 2; ++L) {
        // ---- step A: p at PA = L-1 ----
        const int PA = L - 1;
        const ptrdiff_t colA = (ptrdiff_t)PA * (ptrdiff_t)ld;
        const ptrdiff_t colV0 = (ptrdiff_t)(L - 3) * (ptrdiff_t)ld;
        const float4 xa4 = XF ? make_float4(1.0f, la.kx, 1.0f, la.kx) : __ldg(S.xcoef + (PA + S2D_GX));
        const bool colm = XF || xa4.x == 1.0f;
        const bool pz_live = !(FAST && colm);
        const float4 cvx = ld4(vxi + (ptrdiff_t)L * (ptrdiff_t)ld);
        const float4 cvz = ld4(vzi + colA);
        const float4 cpx = ld4(pxi + colA);
        const float4 cpz = pz_live ? ld4(pzi + colA) : zero;
        const float4 ckk = ld4(kap + colA);
        const float4 cbx = ld4(bxp + colV0);
        const float4 cbz = ld4(bzp + colV0);
        vq0 = vq1; vq1 = vq2; vq2 = vq3;
        vq3 = cvx;
        const float4 vz = cvz;
        float4 pxn, pzn, dxv, dzv;
        const float4 kka = ckk;
        const float4 pn =
            p_update<FAST, XF>(la, S, PA, xa4, colm, vq0, vq1, vq2, vq3, cpx, cpz, kka, vz, pxn, pzn, dxv, dzv);
        const bool in_a = PA >= xa && PA < xb;
        if (TWO) {
            ring_at(ring, 0, PA, lane) = pxn;
            ring_at(ring, 1, PA, lane) = pzn;
        } else if (in_a && la.owner) {
            st4(pxo + colA, pxn);
            if (pz_live) st4(pzo + colA, pzn);
        }
        if (rec_a && in_a) record(la, S, PA, pn, slot_a);
        pq0 = pq1; pq1 = pq2; pq2 = pq3; pq3 = pn;
        zq0 = zq1; zq1 = zq2; zq2 = vz;
        if (L < xaa + 3) continue;
        // ---- step A: v at VA = L-3 ----
        const int VA = L - 3;
        const ptrdiff_t colVA = (ptrdiff_t)VA * (ptrdiff_t)ld;
        float4 vxn, vzn, dxp, dzp;
        const float4 bxa = cbx, bza = cbz;
        v_update<FAST, XF>(la, S, VA, pq0, pq1, pq2, pq3, vq0, zq0, bxa, bza, vxn, vzn, dxp, dzp);
        if (!TWO) {
            if (la.owner) {
                st4(vxo + colVA, vxn);
                st4(vzo + colVA, vzn);
            }
            continue;
        }
        ring_at(ring, 2, VA, lane) = vzn;
        ring_at(ring, 3, VA, lane) = vxn;
        if (L < xa + 3) continue;
        // ---- step B: p at PB = L-4 ----
        const int PB = L - 4;
        const ptrdiff_t colB = (ptrdiff_t)PB * (ptrdiff_t)ld;
        const float4 vzb = ring_at(ring, 2, PB, lane);
        const float4 xb4 = XF ? make_float4(1.0f, lb.kx, 1.0f, lb.kx) : __ldg(S.xcoef + (PB + S2D_GX));
        const bool colmb = XF || xb4.x == 1.0f;
        const bool pz_liveb = !(FAST && colmb);
        float4 pxm, pzm, dxw, dzw;
        const float4 pm = p_update<FAST, XF>(lb, S, PB, xb4, colmb, ring_at(ring, 3, PB - 2, lane),
                                             ring_at(ring, 3, PB - 1, lane),
                                   ring_at(ring, 3, PB, lane), ring_at(ring, 3, PB + 1, lane), ring_at(ring, 0, PB, lane),
                                   pz_liveb ? ring_at(ring, 1, PB, lane) : zero, ld4(kap + colB), vzb,
                                   pxm, pzm, dxw, dzw);
        const bool in_b = PB >= xa && PB < xb;
        if (in_b && la.owner) {
            st4(pxo + colB, pxm);
            if (pz_liveb) st4(pzo + colB, pzm);
        }
        if (rec_b && in_b) record(lb, S, PB, pm, slot_b);
        ring_at(ring, 4, PB, lane) = pm;
        if (L < xa + 6) continue;
        // ---- step B: v at VB = L-6 ----
        const int VB = L - 6;
        const ptrdiff_t colVB = (ptrdiff_t)VB * (ptrdiff_t)ld;
        float4 vxm, vzm, dxq, dzq;
        v_update<FAST, XF>(lb, S, VB, ring_at(ring, 4, VB - 1, lane), ring_at(ring, 4, VB, lane),
                           ring_at(ring, 4, VB + 1, lane),
                 ring_at(ring, 4, VB + 2, lane), ring_at(ring, 3, VB, lane), ring_at(ring, 2, VB, lane),
                 ld4(bxp + colVB), ld4(bzp + colVB), vxm, vzm, dxq, dzq);
        if (la.owner) {
            st4(vxo + colVB, vxm);
            st4(vzo + colVB, vzm);
        }
    }
}

template <bool TWO>
__global__ void __launch_bounds__(128, 4) step_kernel_ts(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + (TWO ? 2 : 1) * kt_off;
    if (kt + (TWO ? 1 : 0) >= a.fd_nt) return;
    const int par = a.par0 ^ (kt_off & 1);
    float4 *ring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kTsWarpBytes);
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        warp_copy_shot(S, G, lane);
        const int c = strip * S2D_TS_OUT - 8;
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
        // columns xa-4 .. xb+4 take part (step A's p reaches xb+4, feeding its v at xb+2)
        const bool xf = xa - 4 >= S.xfast_lo && min(S.nnx, xa + seg_len) + 4 < S.xfast_hi;
        if (zf && xf) ts_task<true, TWO, true>(a, S, strip, xa, seg_len, kt, par, lane, ring);
        else if (zf) ts_task<true, TWO, false>(a, S, strip, xa, seg_len, kt, par, lane, ring);
        else if (xf) ts_task<false, TWO, true>(a, S, strip, xa, seg_len, kt, par, lane, ring);
        else ts_task<false, TWO, false>(a, S, strip, xa, seg_len, kt, par, lane, ring);
    }
}

// ------------------------------------------ 8th-order operator (kVariantO8)
//
// "Order of FD Operator" = 8, which the reference parses but never runs (its
// step exists for 4 only, cpumodelling.cpp:121).  Same scheme, sponge, source
// and receivers as the 4th-order kernels, with the staggered 8th-order
// operators
//   D- f[i] = sum_k c_k (f[i+k-1] - f[i-k]),  D+ f[i] = sum_k c_k (f[i+k] - f[i-k+1]),
// c = (1225/1024, -245/3072, 49/5120, -5/7168), and the reference's 4th-order,
// plain-difference and zero rows where the 8-tap stencil would leave the grid.
//
// One fused pass per step, streamed like the plain-load kernel: the warp keeps
// vx at P-4 .. P+3 (8 columns), new p at V-3 .. V+4 (8 columns) and vz at
// V .. P (5 columns) in registers, forms p at P = L-3 and the velocities at
// V = L-7.  The z-stencils reach 4 rows, one whole neighbouring lane: p is
// exact on lanes 1..30 and the velocities on lanes 2..29, so strips are 112
// rows (the two-step kernel's layout, read from 112k-8) and lanes 2..29 write.

// c1 d1 + c2 d2 + c3 d3 + c4 d4 with the rounding fixed (innermost product
// rounded, then three fused steps).
__device__ __forceinline__ float dif8(const float4 &c, float d1, float d2, float d3, float d4) {
    return __fmaf_rn(c.x, d1, __fmaf_rn(c.y, d2, __fmaf_rn(c.z, d3, __fmul_rn(c.w, d4))));
}
template <bool FAST>
__device__ __forceinline__ float4 zdm8(const Lane<FAST> &ln, int i) {
    if (FAST) return make_float4(kC81, kC82, kC83, kC84);
    return dm8(ln.z0 + i, ln.nnz);
}
template <bool FAST>
__device__ __forceinline__ float4 zdp8(const Lane<FAST> &ln, int i) {
    if (FAST) return make_float4(kC81, kC82, kC83, kC84);
    return dp8(ln.z0 + i, ln.nnz);
}

// New p at column P from vx at P-4 .. P+3 (w), old px, pz, kappa and vz at P;
// the step's first two products (as p_cell forms them) in dxv, dzv.
// XF: column P lies in the 8th-order x-interior (8-tap pair, dampings 1).
template <bool FAST, bool XF = false>
__device__ __forceinline__ float4 p_update8(const Lane<FAST> &ln, const ShotDev &S, int P, const float4 &xc,
                                            bool colm, const float4 (&w)[8], const float4 &px, const float4 &pz,
                                            const float4 &kk, const float4 &vz, float4 &pxn, float4 &pzn,
                                            float4 &dxv, float4 &dzv) {
    // vz rows z0-4 .. z0+6: the lane above's four (u), this lane's, the lane below's first three (d)
    const float u0 = __shfl_up_sync(kFull, vz.x, 1), u1 = __shfl_up_sync(kFull, vz.y, 1);
    const float u2 = __shfl_up_sync(kFull, vz.z, 1), u3 = __shfl_up_sync(kFull, vz.w, 1);
    const float d0 = __shfl_down_sync(kFull, vz.x, 1), d1 = __shfl_down_sync(kFull, vz.y, 1);
    const float d2 = __shfl_down_sync(kFull, vz.z, 1);
    const float dz0 = dif8(zdm8(ln, 0), vz.x - u3, vz.y - u2, vz.z - u1, vz.w - u0);
    const float dz1 = dif8(zdm8(ln, 1), vz.y - vz.x, vz.z - u3, vz.w - u2, d0 - u1);
    const float dz2 = dif8(zdm8(ln, 2), vz.z - vz.y, vz.w - vz.x, d0 - u3, d1 - u2);
    const float dz3 = dif8(zdm8(ln, 3), vz.w - vz.z, d0 - vz.y, d1 - vz.x, d2 - u3);
    const float4 cx = XF ? make_float4(kC81, kC82, kC83, kC84) : dm8(P, S.nnx);
    const float dx0 = dif8(cx, w[4].x - w[3].x, w[5].x - w[2].x, w[6].x - w[1].x, w[7].x - w[0].x);
    const float dx1 = dif8(cx, w[4].y - w[3].y, w[5].y - w[2].y, w[6].y - w[1].y, w[7].y - w[0].y);
    const float dx2 = dif8(cx, w[4].z - w[3].z, w[5].z - w[2].z, w[6].z - w[1].z, w[7].z - w[0].z);
    const float dx3 = dif8(cx, w[4].w - w[3].w, w[5].w - w[2].w, w[6].w - w[1].w, w[7].w - w[0].w);
    const float4 r0 = zrow(ln, 0), r1 = zrow(ln, 1), r2 = zrow(ln, 2), r3 = zrow(ln, 3);
    p_cell(colm && (FAST || r0.x == 1.0f), xc.x, xc.y, r0.x, r0.y, px.x, pz.x, kk.x, dx0, dz0, pxn.x, pzn.x, dxv.x,
           dzv.x);
    p_cell(colm && (FAST || r1.x == 1.0f), xc.x, xc.y, r1.x, r1.y, px.y, pz.y, kk.y, dx1, dz1, pxn.y, pzn.y, dxv.y,
           dzv.y);
    p_cell(colm && (FAST || r2.x == 1.0f), xc.x, xc.y, r2.x, r2.y, px.z, pz.z, kk.z, dx2, dz2, pxn.z, pzn.z, dxv.z,
           dzv.z);
    p_cell(colm && (FAST || r3.x == 1.0f), xc.x, xc.y, r3.x, r3.y, px.w, pz.w, kk.w, dx3, dz3, pxn.w, pzn.w, dxv.w,
           dzv.w);
    if (P == ln.src_x && ln.sdz >= 0 && ln.sdz < 4) {
        if (ln.sdz == 0) pxn.x += ln.amp;
        else if (ln.sdz == 1) pxn.y += ln.amp;
        else if (ln.sdz == 2) pxn.z += ln.amp;
        else pxn.w += ln.amp;
    }
    return make_float4(pxn.x + pzn.x, pxn.y + pzn.y, pxn.z + pzn.z, pxn.w + pzn.w);
}

// Velocities at column V from new p at V-3 .. V+4 (pw), old vx, vz and bx, bz
// at V; D+x p and D+z p in dxp, dzp.
// XF: column V lies in the 8th-order x-interior: no coefficient load.
template <bool FAST, bool XF = false>
__device__ __forceinline__ void v_update8(const Lane<FAST> &ln, const ShotDev &S, int V, const float4 (&pw)[8],
                                          const float4 &vx, const float4 &vz, const float4 &bx, const float4 &bz,
                                          float4 &vxn, float4 &vzn, float4 &dxp, float4 &dzp) {
    const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (V + S2D_GX));
    const float4 cx = XF ? make_float4(kC81, kC82, kC83, kC84) : dp8(V, S.nnx);
    const float ex0 = dif8(cx, pw[4].x - pw[3].x, pw[5].x - pw[2].x, pw[6].x - pw[1].x, pw[7].x - pw[0].x);
    const float ex1 = dif8(cx, pw[4].y - pw[3].y, pw[5].y - pw[2].y, pw[6].y - pw[1].y, pw[7].y - pw[0].y);
    const float ex2 = dif8(cx, pw[4].z - pw[3].z, pw[5].z - pw[2].z, pw[6].z - pw[1].z, pw[7].z - pw[0].z);
    const float ex3 = dif8(cx, pw[4].w - pw[3].w, pw[5].w - pw[2].w, pw[6].w - pw[1].w, pw[7].w - pw[0].w);
    // p rows z0-3 .. z0+7 at V: the lane above's last three (u), this lane's (q), the lane below's four (d)
    const float4 q = pw[3];
    const float u1 = __shfl_up_sync(kFull, q.y, 1), u2 = __shfl_up_sync(kFull, q.z, 1);
    const float u3 = __shfl_up_sync(kFull, q.w, 1);
    const float d0 = __shfl_down_sync(kFull, q.x, 1), d1 = __shfl_down_sync(kFull, q.y, 1);
    const float d2 = __shfl_down_sync(kFull, q.z, 1), d3 = __shfl_down_sync(kFull, q.w, 1);
    const float ez0 = dif8(zdp8(ln, 0), q.y - q.x, q.z - u3, q.w - u2, d0 - u1);
    const float ez1 = dif8(zdp8(ln, 1), q.z - q.y, q.w - q.x, d0 - u3, d1 - u2);
    const float ez2 = dif8(zdp8(ln, 2), q.w - q.z, d0 - q.y, d1 - q.x, d2 - u3);
    const float ez3 = dif8(zdp8(ln, 3), d0 - q.w, d1 - q.z, d2 - q.y, d3 - q.x);
    dxp = make_float4(ex0, ex1, ex2, ex3);
    dzp = make_float4(ez0, ez1, ez2, ez3);
    vxn.x = upd(xc.z, vx.x, xc.w, bx.x, ex0);
    vxn.y = upd(xc.z, vx.y, xc.w, bx.y, ex1);
    vxn.z = upd(xc.z, vx.z, xc.w, bx.z, ex2);
    vxn.w = upd(xc.z, vx.w, xc.w, bx.w, ex3);
    float4 r = zrow(ln, 0);
    vzn.x = upd(r.z, vz.x, r.w, bz.x, ez0);
    r = zrow(ln, 1);
    vzn.y = upd(r.z, vz.y, r.w, bz.y, ez1);
    r = zrow(ln, 2);
    vzn.z = upd(r.z, vz.z, r.w, bz.z, ez2);
    r = zrow(ln, 3);
    vzn.w = upd(r.z, vz.w, r.w, bz.w, ez3);
}

// One (shot, strip, segment) task of the 8th-order step.  Columns read:
// vx at xa-7 .. xb+6, px, pz, kappa, vz at xa-3 .. xb+3, bx, bz at xa .. xb-1
// (inside the 8 ghost columns on each side).
// XF: every column the task updates or differentiates lies in the 8th-order
// x-interior (literal coefficients, no coefficient loads).
template <bool FAST, bool PROD, bool XF = false>
__device__ __forceinline__ void o8_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len, int kt,
                                        int par, bool rec_step, int slot, int lane) {
    const int xb = min(S.nnx, xa + seg_len);
    const size_t ld = (size_t)S.ld;
    const int c = strip * S2D_TS_OUT - 8;
    Lane<FAST> ln;
    lane_setup(ln, S, c, lane, kt);
    ln.owner = lane >= 2 && lane <= 29 && ln.z0 >= 0 && ln.z0 < S.nnz;
    // receivers only where the strip's rows hold some
    const bool rec = rec_step && slot < S.real_nt && !(a.flags & S2D_STEP_NO_RECORD) &&
                     c + S2D_STRIP_ROWS > S.rec_zlo && c <= S.rec_zhi;
    const size_t off = (size_t)(ln.z0 + S2D_GZ) + (size_t)S2D_GX * ld;
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off;
    const int ib = par * 4 * fs, ob = (par ^ 1) * 4 * fs;
    const float *__restrict__ pxi = sb + ib;
    const float *__restrict__ pzi = sb + ib + fs;
    const float *__restrict__ vxi = sb + ib + 2 * fs;
    const float *__restrict__ vzi = sb + ib + 3 * fs;
    float *__restrict__ pxo = sb + ob;
    float *__restrict__ pzo = sb + ob + fs;
    float *__restrict__ vxo = sb + ob + 2 * fs;
    float *__restrict__ vzo = sb + ob + 3 * fs;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = kap + fs;
    const float *__restrict__ bzp = kap + 2 * fs;
    const size_t F = (size_t)(S.nnx + 2 * S2D_GX) * ld;
    float *__restrict__ pr = PROD ? S.prod + (size_t)(kt - a.prod_kt0) * 4 * F + off : nullptr;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 w[8], pw[8], zq[5];
#pragma unroll
    for (int i = 0; i < 8; ++i) pw[i] = zero;
#pragma unroll
    for (int i = 0; i < 5; ++i) zq[i] = zero;
    w[0] = zero;
#pragma unroll
    for (int i = 1; i < 8; ++i) w[i] = ld4(vxi + (ptrdiff_t)(xa - 8 + i) * (ptrdiff_t)ld);
    for (int L = xa; L <= xb + 6; ++L) {
        const int P = L - 3;
        const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
#pragma unroll
        for (int i = 0; i < 7; ++i) w[i] = w[i + 1];
        w[7] = ld4(vxi + (ptrdiff_t)L * (ptrdiff_t)ld);
        const float4 vz = ld4(vzi + colP);
        const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
        const bool colm = XF || xc.x == 1.0f;
        const bool pz_live = !(FAST && colm);
        float4 pxn, pzn, dxv, dzv;
        const float4 pn = p_update8<FAST, XF>(ln, S, P, xc, colm, w, ld4(pxi + colP),
                                              pz_live ? ld4(pzi + colP) : zero, ld4(kap + colP), vz, pxn, pzn,
                                              dxv, dzv);
        const bool in_seg = P >= xa && P < xb;
        if (in_seg && ln.owner) {
            st4(pxo + colP, pxn);
            if (pz_live) st4(pzo + colP, pzn);
            if (PROD) {
                st4(pr + colP, dxv);
                if (pz_live) st4(pr + F + colP, dzv);
            }
        }
        if (rec && in_seg) record(ln, S, P, pn, slot);
#pragma unroll
        for (int i = 0; i < 7; ++i) pw[i] = pw[i + 1];
        pw[7] = pn;
#pragma unroll
        for (int i = 0; i < 4; ++i) zq[i] = zq[i + 1];
        zq[4] = vz;
        if (L >= xa + 7) {
            const int V = L - 7;
            const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
            float4 vxn, vzn, dxp, dzp;
            v_update8<FAST, XF>(ln, S, V, pw, w[0], zq[0], ld4(bxp + colV), ld4(bzp + colV), vxn, vzn, dxp, dzp);
            if (ln.owner) {
                st4(vxo + colV, vxn);
                st4(vzo + colV, vzn);
                if (PROD) {
                    st4(pr + 2 * F + colV, dxp);
                    st4(pr + 3 * F + colV, dzp);
                }
            }
        }
    }
}

// The same task with its windows in a per-warp shared-memory ring instead of
// registers (kVariantO8s, 128 registers, 16 warps per SM): vx of the last 8
// columns, new p of the last 8, vz of the last 4.  Each lane reads back only
// the entries it wrote, so the ring needs no synchronisation.
__device__ __forceinline__ float4 &o8_ring(float4 *ring, int field, int col, int lane) {
    // field 0: vx (8 slots), 1: new p (8 slots), 2: vz (4 slots)
    return field == 2 ? ring[(16 + (col & 3)) * 32 + lane] : ring[(field * 8 + (col & 7)) * 32 + lane];
}

// XF: as for o8_task, literal column coefficients on x-interior tasks.
template <bool FAST, bool XF = false>
__device__ __forceinline__ void o8s_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len, int kt,
                                         int par, bool rec_step, int slot, int lane, float4 *ring) {
    const int xb = min(S.nnx, xa + seg_len);
    const size_t ld = (size_t)S.ld;
    const int c = strip * S2D_TS_OUT - 8;
    Lane<FAST> ln;
    lane_setup(ln, S, c, lane, kt);
    ln.owner = lane >= 2 && lane <= 29;
    // receivers only where the strip's rows hold some
    const bool rec = rec_step && slot < S.real_nt && !(a.flags & S2D_STEP_NO_RECORD) &&
                     c + S2D_STRIP_ROWS > S.rec_zlo && c <= S.rec_zhi;
    const size_t off = (size_t)(ln.z0 + S2D_GZ) + (size_t)S2D_GX * ld;
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off;
    const int ib = par * 4 * fs, ob = (par ^ 1) * 4 * fs;
    const float *__restrict__ pxi = sb + ib;
    const float *__restrict__ pzi = sb + ib + fs;
    const float *__restrict__ vxi = sb + ib + 2 * fs;
    const float *__restrict__ vzi = sb + ib + 3 * fs;
    float *__restrict__ pxo = sb + ob;
    float *__restrict__ pzo = sb + ob + fs;
    float *__restrict__ vxo = sb + ob + 2 * fs;
    float *__restrict__ vzo = sb + ob + 3 * fs;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = kap + fs;
    const float *__restrict__ bzp = kap + 2 * fs;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int col = xa - 7; col < xa; ++col) o8_ring(ring, 0, col, lane) = ld4(vxi + (ptrdiff_t)col * (ptrdiff_t)ld);
    for (int L = xa; L <= xb + 6; ++L) {
        const int P = L - 3;
        const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
        float4 w[8];
        w[7] = ld4(vxi + (ptrdiff_t)L * (ptrdiff_t)ld);
#pragma unroll
        for (int i = 0; i < 7; ++i) w[i] = o8_ring(ring, 0, L - 7 + i, lane);
        o8_ring(ring, 0, L, lane) = w[7];  // the slot of column L-8, no longer needed
        const float4 vz = ld4(vzi + colP);
        const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
        const bool colm = XF || xc.x == 1.0f;
        const bool pz_live = !(FAST && colm);
        float4 pxn, pzn, dxv, dzv;
        const float4 pn = p_update8<FAST, XF>(ln, S, P, xc, colm, w, ld4(pxi + colP),
                                              pz_live ? ld4(pzi + colP) : zero, ld4(kap + colP), vz, pxn, pzn, dxv,
                                              dzv);
        const bool in_seg = P >= xa && P < xb;
        if (in_seg && ln.owner) {
            st4(pxo + colP, pxn);
            if (pz_live) st4(pzo + colP, pzn);
        }
        if (rec && in_seg) record(ln, S, P, pn, slot);
        const float4 vzV = o8_ring(ring, 2, P - 4, lane);  // read before vz at P takes its slot
        o8_ring(ring, 2, P, lane) = vz;
        o8_ring(ring, 1, P, lane) = pn;                    // the slot of column P-8
        if (L >= xa + 7) {
            const int V = L - 7;
            const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
            float4 pw[8];
#pragma unroll
            for (int i = 0; i < 7; ++i) pw[i] = o8_ring(ring, 1, V - 3 + i, lane);
            pw[7] = pn;
            float4 vxn, vzn, dxp, dzp;
            v_update8<FAST, XF>(ln, S, V, pw, w[0], vzV, ld4(bxp + colV), ld4(bzp + colV), vxn, vzn, dxp, dzp);
            if (ln.owner) {
                st4(vxo + colV, vxn);
                st4(vzo + colV, vzn);
            }
        }
    }
}

// Debug self-check (S2D_DEVICE_CHECKS) of the 8th-order task's reach.
__device__ __forceinline__ bool o8_in_bounds(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len) {
#ifdef S2D_DEVICE_CHECKS
    const long ld = S.ld;
    const int xb = min(S.nnx, xa + seg_len);
    const long c = (long)strip * S2D_TS_OUT - 8;
    const long F = (long)(S.nnx + 2 * S2D_GX) * ld;
    const long lo = (long)(xa - 7 + S2D_GX) * ld + (c + S2D_GZ);
    const long hi = (long)(xb + 6 + S2D_GX) * ld + (c + S2D_GZ) + 127;
    if (xa - 7 < -S2D_GX || xb + 6 >= S.nnx + S2D_GX || c + S2D_GZ < 0 || c + 127 + S2D_GZ >= ld || lo < 0 ||
        hi >= F || (size_t)F > S.nfield) {
        if (a.err) atomicCAS(a.err, 0, (3 << 8) | 1);
        return false;
    }
#endif
    return true;
}

// MINB blocks of 4 warps per SM: 3 caps registers at 168 (some spill), 2
// leaves the 224 the windows (84 registers) and stencils need.
template <int MINB, bool PROD>
__global__ void __launch_bounds__(128, MINB) step_kernel_o8(const StepArgs *__restrict__ A, int kt_off) {
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    const int par = a.par0 ^ (kt_off & 1);
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        warp_copy_shot(S, G, lane);
        if (!o8_in_bounds(a, S, strip, xa, seg_len)) continue;
        const int c = strip * S2D_TS_OUT - 8;
        // literal coefficients: every row of the strip 8th-order and undamped in z
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1) && c >= 4 && c + S2D_STRIP_ROWS - 1 <= S.nnz - 5;
        // pressure on columns xa-3 .. xb+3 (8-tap D-: columns [4, nnx-4]),
        // velocities on xa .. xb-1 (D+: [3, nnx-5]), all undamped in x
        const int xb = min(S.nnx, xa + seg_len);
        const bool xf = xa - 3 >= max(S.xfast_lo, 4) && xb + 3 < min(S.xfast_hi, S.nnx - 3);
        if (zf && xf) o8_task<true, PROD, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else if (zf) o8_task<true, PROD, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else if (xf) o8_task<false, PROD, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
        else o8_task<false, PROD, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane);
    }
}

// The shared-memory-ring form: 128 registers, 4 blocks of 4 warps per SM,
// kO8sWarpBytes of dynamic shared memory per warp.
__global__ void __launch_bounds__(128, 4) step_kernel_o8s(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    float4 *ring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kO8sWarpBytes);
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    const int par = a.par0 ^ (kt_off & 1);
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        warp_copy_shot(S, G, lane);
        if (!o8_in_bounds(a, S, strip, xa, seg_len)) continue;
        const int c = strip * S2D_TS_OUT - 8;
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1) && c >= 4 && c + S2D_STRIP_ROWS - 1 <= S.nnz - 5;
        // the columns of o8_task's x-interior condition
        const int xb = min(S.nnx, xa + seg_len);
        const bool xf = xa - 3 >= max(S.xfast_lo, 4) && xb + 3 < min(S.xfast_hi, S.nnx - 3);
        if (zf && xf) o8s_task<true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else if (zf) o8s_task<true, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else if (xf) o8s_task<false, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else o8s_task<false, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
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

// ------------------------------------------------------------ async variant
//
// The plain-load kernel's loop with every column load replaced by a per-lane
// asynchronous copy (cp.async, 16 bytes: the lane's four rows) into a
// per-warp ring of kAsyncStages iterations in shared memory, issued
// kAsyncStages - 1 iterations ahead: the loads of the next columns are in
// flight while the warp computes, without holding registers.  Each lane reads
// back only the 16 bytes it copied itself (z-neighbours still come by
// shuffles), so the ring needs no barrier: cp.async.wait_group on the lane's
// own copy groups is the whole synchronisation.  A ghost lane's copies are
// zero-fills that read nothing.  The arithmetic is ldg_task's: the same bits.


template <bool PROD, bool FAST, bool XF>
__device__ __forceinline__ void async_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len,
                                           int kt, int par, bool rec_step, int slot, int lane, float4 *ring) {
    const int xb = min(S.nnx, xa + seg_len);
    const size_t ld = (size_t)S.ld;
    const int c = strip * S2D_STRIP_OUT - 4;
    Lane<FAST> ln;
    lane_setup(ln, S, c, lane, kt);
    const bool ghost = ln.z0 < 0 || ln.z0 >= S.nnz;
    const bool rec = rec_step && slot < S.real_nt && !(a.flags & S2D_STEP_NO_RECORD) &&
                     c + S2D_STRIP_ROWS > S.rec_zlo && c <= S.rec_zhi;
    const size_t off = (size_t)(ln.z0 + S2D_GZ) + (size_t)S2D_GX * ld;
    const size_t F = (size_t)(S.nnx + 2 * S2D_GX) * ld;
    float *__restrict__ pr = PROD ? S.prod + (size_t)(kt - a.prod_kt0) * 4 * F + off : nullptr;
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off;
    const int ib = par * 4 * fs, ob = (par ^ 1) * 4 * fs;
    const float *pxi = sb + ib;
    const float *pzi = sb + ib + fs;
    const float *vxi = sb + ib + 2 * fs;
    const float *vzi = sb + ib + 3 * fs;
    float *__restrict__ pxo = sb + ob;
    float *__restrict__ pzo = sb + ob + fs;
    float *__restrict__ vxo = sb + ob + 2 * fs;
    float *__restrict__ vzo = sb + ob + 3 * fs;
    const float *kap = S.kappa + off;
    const float *bxp = kap + fs;
    const float *bzp = kap + 2 * fs;
    // iteration i = 0 .. n_it-1 is column L = xa-3+i; its slots: vx at L,
    // px, pz, kappa, vz at L-1, bx, bz at L-3 (ring float4 index
    // ((i % kAsyncStages) * kAsyncSlots + f) * 32 + lane)
    const int n_it = xb - xa + 6;
    auto issue = [&](int i) {
        float4 *st = ring + (i % kAsyncStages) * kAsyncSlots * 32 + lane;
        const int L = xa - 3 + i;
        const ptrdiff_t cL = (ptrdiff_t)L * (ptrdiff_t)ld, cP = cL - (ptrdiff_t)ld, cV = cL - 3 * (ptrdiff_t)ld;
        const bool live = !ghost;
        cp_async16(st, vxi + cL, live);
        if (L >= xa) {
            const bool pz_live = !(FAST && (XF || __ldg(S.xcoef + (L - 1 + S2D_GX)).x == 1.0f));
            cp_async16(st + 1 * 32, pxi + cP, live);
            if (pz_live) cp_async16(st + 2 * 32, pzi + cP, live);
            cp_async16(st + 3 * 32, kap + cP, live);
            cp_async16(st + 4 * 32, vzi + cP, live);
        }
        if (L >= xa + 3) {
            cp_async16(st + 5 * 32, bxp + cV, live);
            cp_async16(st + 6 * 32, bzp + cV, live);
        }
    };
#pragma unroll
    for (int i = 0; i < kAsyncStages - 1; ++i) {
        if (i < n_it) issue(i);
        cp_async_commit();
    }
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 vq0 = zero, vq1 = zero, vq2 = zero, vq3 = zero;
    float4 pq0 = zero, pq1 = zero, pq2 = zero, pq3 = zero;
    float4 zq0 = zero, zq1 = zero, zq2 = zero;
    for (int i = 0; i < n_it; ++i) {
        if (i + kAsyncStages - 1 < n_it) issue(i + kAsyncStages - 1);
        cp_async_commit();
        cp_async_wait<kAsyncStages - 1>();  // iteration i's copies have landed
        const float4 *st = ring + (i % kAsyncStages) * kAsyncSlots * 32 + lane;
        const int L = xa - 3 + i;
        vq0 = vq1; vq1 = vq2; vq2 = vq3;
        vq3 = st[0];
        if (L < xa) continue;
        const int P = L - 1;
        const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
        const float4 vz = st[4 * 32];
        const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
        const bool colm = XF || xc.x == 1.0f;
        const bool pz_live = !(FAST && colm);
        float4 pxn, pzn, dxv, dzv;
        const float4 pn = p_update<FAST, XF>(ln, S, P, xc, colm, vq0, vq1, vq2, vq3, st[1 * 32],
                                             pz_live ? st[2 * 32] : zero, st[3 * 32], vz, pxn, pzn, dxv, dzv);
        const bool in_seg = P >= xa && P < xb;
        if (in_seg && ln.owner) {
            st4(pxo + colP, pxn);
            if (pz_live) st4(pzo + colP, pzn);
            if (PROD) {
                st4(pr + colP, dxv);
                if (pz_live) st4(pr + F + colP, dzv);
            }
        }
        if (rec && in_seg) record(ln, S, P, pn, slot);
        pq0 = pq1; pq1 = pq2; pq2 = pq3; pq3 = pn;
        zq0 = zq1; zq1 = zq2; zq2 = vz;
        if (L >= xa + 3) {
            const int V = L - 3;
            const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
            float4 vxn, vzn, dxp, dzp;
            v_update<FAST, XF>(ln, S, V, pq0, pq1, pq2, pq3, vq0, zq0, st[5 * 32], st[6 * 32], vxn, vzn, dxp, dzp);
            if (ln.owner) {
                st4(vxo + colV, vxn);
                st4(vzo + colV, vzn);
                if (PROD) {
                    st4(pr + 2 * F + colV, dxp);
                    st4(pr + 3 * F + colV, dzp);
                }
            }
        }
    }
    cp_async_wait<0>();
}

template <bool PROD, int MINB>
__global__ void __launch_bounds__(128, MINB) step_kernel_async(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    float4 *ring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kAsyncWarpBytes);
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    const int par = a.par0 ^ (kt_off & 1);
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        warp_copy_shot(S, G, lane);
        if (!task_in_bounds(a, S, strip, xa, seg_len, kt, PROD, 1)) continue;
        const int c = strip * S2D_STRIP_OUT - 4;
        const int xb = min(S.nnx, xa + seg_len);
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
        const bool xf = xa - 1 >= S.xfast_lo && xb + 1 < S.xfast_hi;
        if (zf && xf) async_task<PROD, true, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else if (zf) async_task<PROD, true, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else if (xf) async_task<PROD, false, true>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
        else async_task<PROD, false, false>(a, S, strip, xa, seg_len, kt, par, rec_step, slot, lane, ring);
    }
}

// ---------------------------------------------------------------- TMA variant
//
// A CTA is kTmaWarps consumer warps and one producer warp.  A task is one
// x-segment of kTmaWarps consecutive (shot, strip) pairs of a model group
// (consecutive strips of one shot, wrapping into the next shot), so the
// consumer warps of a CTA stream adjacent 128-row strips of the same columns.
// The producer brings the columns in as 2-D tensor boxes (128 rows x kTmaCols
// columns, cp.async.bulk.tensor from this GPU's own memory, no multicast)
// into a kTmaStages-deep ring in shared memory, one full barrier (transaction
// bytes) and one empty barrier (one arrival per consumer warp) per stage, so
// that up to kTmaStages * kTmaStageBytes of loads are in flight per SM while
// the consumer warps compute from shared memory.  Stage k of a task holds, for
// the consumer iterations L = xa-3+2k and L+1 (the loop of ldg_task), vx at L,
// px, pz, kappa, vz at L-1 and bx, bz at L-3; boxes a task does not need are
// not loaded, nor pz where every cell of both columns carries p alone.  The
// tensor maps end at row nnz of the grid: the rows of the last strip past the
// grid arrive as zeros (the ghost rows hold zeros) without DRAM traffic.  The
// update arithmetic is ldg_task's (p_update, v_update, record): the same bits.
//
// Every wait is bounded (StepArgs::spin_limit polls).  A consumer that gives
// up records S2D_DEV_ERR_WAIT and leaves; the producer, when its own wait for
// a free stage gives up, stops issuing, records the error and waits (bounded)
// for its copies in flight before it leaves, so no copy lands in released
// shared memory.

__device__ __forceinline__ void tma_load_3d(void *dst, const void *map, int z, int x, int plane, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(z), "r"(x), "r"(plane), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// The (shot, strip) pair consumer warp w of task t works on.
struct TmaPair {
    int group, shot, strip, xa, seg_len;
    bool live;  // false when the task's block has fewer pairs than warps
};
__device__ __forceinline__ TmaPair tma_pair(const StepArgs &a, int t, int w) {
    int g = 0;
    while (g + 1 < a.ngroups && __ldg(&a.groups[g + 1].task_begin) <= t) ++g;
    const GroupDev &G = a.groups[g];
    const int nblk = tma_blocks(G.nshots, G.nstrips);
    const int tl = t - G.task_begin;
    const int p = (tl % nblk) * kTmaWarps + w;
    TmaPair r;
    r.group = g;
    r.live = p < G.nshots * G.nstrips;
    r.shot = G.shot0 + (r.live ? p / G.nstrips : 0);
    r.strip = r.live ? p % G.nstrips : 0;
    r.seg_len = G.seg_len;
    r.xa = (tl / nblk) * G.seg_len;
    return r;
}
// Consumer iterations of a task (L = xa-3 .. xb+2) in stages of kTmaCols.
__device__ __forceinline__ int tma_stages(int xa, int xb) { return (xb - xa + 6 + kTmaCols - 1) / kTmaCols; }

// Producer warp: lane w < kTmaWarps issues the boxes of consumer warp w.
__device__ void tma_produce(const StepArgs &a, int par, unsigned char *ring, uint64_t *full, uint64_t *empty,
                            int lane) {
    const char *maps = static_cast<const char *>(a.tmaps);
    const int drain_limit = a.spin_limit < kDrainLimit / 64 ? a.spin_limit * 64 : kDrainLimit;
    unsigned ph_of[kTmaStages];
    bool pending[kTmaStages];
#pragma unroll
    for (int i = 0; i < kTmaStages; ++i) {
        ph_of[i] = 0;
        pending[i] = false;
    }
    int s = 0, it = 0;
    unsigned ph = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < a.total_tasks && ok; t += gridDim.x) {
        const TmaPair pr = tma_pair(a, t, lane < kTmaWarps ? lane : 0);
        const bool mine = lane < kTmaWarps && pr.live;
        const ShotDev &S = a.shots[pr.shot];
        const int xa = pr.xa, xb = min(S.nnx, xa + pr.seg_len);
        const int nst = tma_stages(xa, xb);
        const int c = pr.strip * S2D_STRIP_OUT - 4;
        const int z = c + S2D_GZ;
        const bool fast = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
        const bool xf = xa - 1 >= S.xfast_lo && xb + 1 < S.xfast_hi;  // every column merged in x
        const void *smap = maps + (size_t)pr.shot * kTmaMapBytes;
        const void *mmap = maps + (size_t)(a.tmap_mat0 + pr.shot) * kTmaMapBytes;
        for (int k = 0; k < nst; ++k, ++it) {
            const int L0 = xa - 3 + kTmaCols * k;
            const bool pbox = L0 >= xa - 1 && L0 <= xb + 2;
            const bool bbox = L0 >= xa + 2 && L0 <= xb + 2;
            bool pz = false;
            if (mine && pbox) {
                pz = !fast;
                if (!pz && !xf) {
#pragma unroll
                    for (int j = 0; j < kTmaCols; ++j) pz = pz || __ldg(S.xcoef + (L0 - 1 + j + S2D_GX)).x != 1.0f;
                }
            }
            unsigned bytes =
                mine ? (unsigned)kTmaBoxBytes * (1u + (pbox ? 3u + (pz ? 1u : 0u) : 0u) + (bbox ? 2u : 0u)) : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(kFull, bytes, o);
            // a free stage: its previous contents consumed by every consumer warp
            bool got = false;
            if (lane == 0) {
                for (int i = 0; i < a.spin_limit && !got; ++i) got = mbar_try_wait(&empty[s], ph ^ 1u);
                if (got) mbar_expect_tx(&full[s], bytes);
            }
            got = __shfl_sync(kFull, got, 0);
            if (!got) {
                ok = false;
                break;
            }
            __syncwarp();
            if (mine && it != a.fault_iter) {
                unsigned char *st = ring + (size_t)s * kTmaStageBytes + (size_t)lane * kTmaBoxBytes;
                const int pa = par * 4;
                tma_load_3d(st, smap, z, L0 + S2D_GX, pa + 2, &full[s]);  // vx
                if (pbox) {
                    const int xp = L0 - 1 + S2D_GX;
                    tma_load_3d(st + 1 * kTmaWarps * kTmaBoxBytes, smap, z, xp, pa + 0, &full[s]);  // px
                    if (pz) tma_load_3d(st + 2 * kTmaWarps * kTmaBoxBytes, smap, z, xp, pa + 1, &full[s]);
                    tma_load_3d(st + 3 * kTmaWarps * kTmaBoxBytes, mmap, z, xp, 0, &full[s]);       // kappa
                    tma_load_3d(st + 4 * kTmaWarps * kTmaBoxBytes, smap, z, xp, pa + 3, &full[s]);  // vz
                }
                if (bbox) {
                    const int xv = L0 - 3 + S2D_GX;
                    tma_load_3d(st + 5 * kTmaWarps * kTmaBoxBytes, mmap, z, xv, 1, &full[s]);  // bx
                    tma_load_3d(st + 6 * kTmaWarps * kTmaBoxBytes, mmap, z, xv, 2, &full[s]);  // bz
                }
            }
            ph_of[s] = ph;
            pending[s] = true;
            if (++s == kTmaStages) {
                s = 0;
                ph ^= 1u;
            }
        }
    }
    if (lane != 0) return;
    if (!ok) atomicOr(a.err, S2D_DEV_ERR_WAIT);
    // copies still in flight must land before the CTA's shared memory is released
#pragma unroll
    for (int i = 0; i < kTmaStages; ++i) {
        if (!pending[i]) continue;
        bool done = false;
        for (int n = 0; n < drain_limit && !done; ++n) done = mbar_try_wait(&full[i], ph_of[i]);
        if (!done) atomicOr(a.err, S2D_DEV_ERR_DRAIN);
    }
}

// One task of a consumer warp; returns false when a wait gave up.  XF: every
// column the task updates or differentiates lies in the shot's x-interior.
template <bool PROD, bool FAST, bool XF>
__device__ __forceinline__ bool tma_task(const StepArgs &a, const ShotDev &S, const TmaPair &pr, int kt, int par,
                                         bool rec_step, int slot, int warp, int lane, const unsigned char *ring,
                                         uint64_t *full, uint64_t *empty, int &s, unsigned &ph) {
    const int xa = pr.xa, xb = min(S.nnx, xa + pr.seg_len);
    const int nst = tma_stages(xa, xb);
    const size_t ld = (size_t)S.ld;
    const int c = pr.strip * S2D_STRIP_OUT - 4;
    Lane<FAST> ln;
    lane_setup(ln, S, c, lane, kt);
    // receivers only where the strip's rows hold some
    const bool rec = pr.live && rec_step && slot < S.real_nt && !(a.flags & S2D_STEP_NO_RECORD) &&
                     c + S2D_STRIP_ROWS > S.rec_zlo && c <= S.rec_zhi;
    const size_t off = (size_t)(ln.z0 + S2D_GZ) + (size_t)S2D_GX * ld;
    const size_t F = (size_t)(S.nnx + 2 * S2D_GX) * ld;
    float *__restrict__ pr_ = PROD ? S.prod + (size_t)(kt - a.prod_kt0) * 4 * F + off : nullptr;
    const int fs = S.fstride;
    float *const sb = S.st[0][0] + off + (par ^ 1) * 4 * fs;
    float *__restrict__ pxo = sb;
    float *__restrict__ pzo = sb + fs;
    float *__restrict__ vxo = sb + 2 * fs;
    float *__restrict__ vzo = sb + 3 * fs;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 vq0 = zero, vq1 = zero, vq2 = zero, vq3 = zero;
    float4 pq0 = zero, pq1 = zero, pq2 = zero, pq3 = zero;
    float4 zq0 = zero, zq1 = zero, zq2 = zero;
    for (int k = 0; k < nst; ++k) {
        if (!wait_stage(&full[s], ph, a.spin_limit)) {
            if (lane == 0) atomicOr(a.err, S2D_DEV_ERR_WAIT);
            return false;
        }
        if (pr.live) {
            const float4 *stg =
                reinterpret_cast<const float4 *>(ring + (size_t)s * kTmaStageBytes + (size_t)warp * kTmaBoxBytes) +
                lane;
            // slot f, column j of the stage: float4 index (f * kTmaWarps * kTmaCols + j) * 32 past stg
#pragma unroll
            for (int j = 0; j < kTmaCols; ++j) {
                const int L = xa - 3 + kTmaCols * k + j;
                if (L > xb + 2) break;
                auto slotv = [&](int f) { return stg[(f * kTmaWarps * kTmaCols + j) * 32]; };
                vq0 = vq1; vq1 = vq2; vq2 = vq3;
                vq3 = slotv(0);
                if (L < xa) continue;
                const int P = L - 1;
                const ptrdiff_t colP = (ptrdiff_t)P * (ptrdiff_t)ld;
                const float4 vz = slotv(4);
                const float4 xc = XF ? make_float4(1.0f, ln.kx, 1.0f, ln.kx) : __ldg(S.xcoef + (P + S2D_GX));
                const bool colm = XF || xc.x == 1.0f;
                const bool pz_live = !(FAST && colm);
                float4 pxn, pzn, dxv, dzv;
                const float4 pn = p_update<FAST, XF>(ln, S, P, xc, colm, vq0, vq1, vq2, vq3, slotv(1),
                                                     pz_live ? slotv(2) : zero, slotv(3), vz, pxn, pzn, dxv, dzv);
                const bool in_seg = P >= xa && P < xb;
                if (in_seg && ln.owner) {
                    st4(pxo + colP, pxn);
                    if (pz_live) st4(pzo + colP, pzn);
                    if (PROD) {
                        st4(pr_ + colP, dxv);
                        if (pz_live) st4(pr_ + F + colP, dzv);
                    }
                }
                if (rec && in_seg) record(ln, S, P, pn, slot);
                pq0 = pq1; pq1 = pq2; pq2 = pq3; pq3 = pn;
                zq0 = zq1; zq1 = zq2; zq2 = vz;
                if (L >= xa + 3) {
                    const int V = L - 3;
                    const ptrdiff_t colV = (ptrdiff_t)V * (ptrdiff_t)ld;
                    float4 vxn, vzn, dxp, dzp;
                    v_update<FAST, XF>(ln, S, V, pq0, pq1, pq2, pq3, vq0, zq0, slotv(5), slotv(6), vxn, vzn, dxp,
                                       dzp);
                    if (ln.owner) {
                        st4(vxo + colV, vxn);
                        st4(vzo + colV, vzn);
                        if (PROD) {
                            st4(pr_ + 2 * F + colV, dxp);
                            st4(pr_ + 3 * F + colV, dzp);
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (++s == kTmaStages) {
            s = 0;
            ph ^= 1u;
        }
    }
    return true;
}

template <bool PROD>
__global__ void __launch_bounds__(kTmaThreads, 1) step_kernel_tma(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ unsigned char smem_raw[];
    // the boxes need 128-byte aligned destinations: align the ring to 1 KB
    unsigned char *ring = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)kTmaStages * kTmaStageBytes);
    uint64_t *empty = full + kTmaStages;
    const StepArgs a = *A;
    const int kt = a.kt_base + kt_off;
    if (kt >= a.fd_nt) return;
    // an earlier launch of this sequence gave up: its wavefields are not valid
    if (*reinterpret_cast<volatile int *>(a.err) != 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kTmaStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kTmaWarps);
        }
        fence_mbar_init();
    }
    __syncthreads();
    const int par = a.par0 ^ (kt_off & 1);
    if (warp == kTmaWarps) {
        tma_produce(a, par, ring, full, empty, lane);
        return;
    }
    const bool rec_step = ((kt + 1) % a.dt_factor) == 0;
    const int slot = (kt + 1) / a.dt_factor - 1;
    int s = 0;
    unsigned ph = 0;
    for (int t = blockIdx.x; t < a.total_tasks; t += gridDim.x) {
        const TmaPair pr = tma_pair(a, t, warp);
        const ShotDev &S = a.shots[pr.shot];
        const int c = pr.strip * S2D_STRIP_OUT - 4;
        const int xa = pr.xa, xb = min(S.nnx, xa + pr.seg_len);
        const bool zf = rows_fast(S, c, c + S2D_STRIP_ROWS - 1);
        // columns xa-1 .. xb+1 take part (p there, v on xa .. xb-1)
        const bool xf = xa - 1 >= S.xfast_lo && xb + 1 < S.xfast_hi;
        bool ok;
        if (zf && xf)
            ok = tma_task<PROD, true, true>(a, S, pr, kt, par, rec_step, slot, warp, lane, ring, full, empty, s, ph);
        else if (zf)
            ok = tma_task<PROD, true, false>(a, S, pr, kt, par, rec_step, slot, warp, lane, ring, full, empty, s, ph);
        else if (xf)
            ok = tma_task<PROD, false, true>(a, S, pr, kt, par, rec_step, slot, warp, lane, ring, full, empty, s, ph);
        else
            ok = tma_task<PROD, false, false>(a, S, pr, kt, par, rec_step, slot, warp, lane, ring, full, empty, s, ph);
        if (!ok) return;
    }
}

}  // namespace

int launch_step(int variant, const StepArgs *args_dev, int kt_off, int grid, int block, size_t smem,
                void *stream) {
    if (variant == kVariantBulk)
        step_kernel_bulk<1><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantBulk128)
        step_kernel_bulk<4><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgProducts)
        step_kernel_ldg<true, 3><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdg128)
        step_kernel_ldg<false, 4><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantTs2)
        step_kernel_ts<true><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantTs1)
        step_kernel_ts<false><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantO8)
        step_kernel_o8<3, false><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantO8r)
        step_kernel_o8<2, false><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantO8Products)
        step_kernel_o8<3, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantO8s)
        step_kernel_o8s<<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantTma)
        step_kernel_tma<false><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantAsync)
        step_kernel_async<false, 4><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgU4)
        step_kernel_ldg<false, 4, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgPf)
        step_kernel_ldg<false, 3, false, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgPf4)
        step_kernel_ldg<false, 4, false, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgPfU4)
        step_kernel_ldg<false, 4, true, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgPfU3)
        step_kernel_ldg<false, 3, true, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantLdgPfProducts)
        step_kernel_ldg<true, 3, false, true><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    else if (variant == kVariantAsyncProducts)
        step_kernel_async<true, 3><<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    else
        step_kernel_ldg<false, 1><<<grid, block, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    return (int)cudaGetLastError();
}

int launch_persist(const StepArgs *args_dev, int nsteps, unsigned *bar, int grid, void *stream) {
    void *args[] = {(void *)&args_dev, (void *)&nsteps, (void *)&bar};
    return (int)cudaLaunchCooperativeKernel((const void *)step_kernel_persist<4>, dim3(grid), dim3(128), args, 0,
                                            (cudaStream_t)stream);
}

int persist_occupancy(int *blocks_per_sm) {
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, step_kernel_persist<4>, 128, 0);
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

namespace {
const void *kernel_of(int variant) {
    if (variant == kVariantBulk) return (const void *)step_kernel_bulk<1>;
    if (variant == kVariantBulk128) return (const void *)step_kernel_bulk<4>;
    if (variant == kVariantLdgProducts) return (const void *)step_kernel_ldg<true, 3>;
    if (variant == kVariantLdg128) return (const void *)step_kernel_ldg<false, 4>;
    if (variant == kVariantTs2) return (const void *)step_kernel_ts<true>;
    if (variant == kVariantTs1) return (const void *)step_kernel_ts<false>;
    if (variant == kVariantO8) return (const void *)step_kernel_o8<3, false>;
    if (variant == kVariantO8r) return (const void *)step_kernel_o8<2, false>;
    if (variant == kVariantO8Products) return (const void *)step_kernel_o8<3, true>;
    if (variant == kVariantO8s) return (const void *)step_kernel_o8s;
    if (variant == kVariantTma) return (const void *)step_kernel_tma<false>;
    if (variant == kVariantAsync) return (const void *)step_kernel_async<false, 4>;
    if (variant == kVariantLdgU4) return (const void *)step_kernel_ldg<false, 4, true>;
    if (variant == kVariantLdgPf) return (const void *)step_kernel_ldg<false, 3, false, true>;
    if (variant == kVariantLdgPf4) return (const void *)step_kernel_ldg<false, 4, false, true>;
    if (variant == kVariantLdgPfU4) return (const void *)step_kernel_ldg<false, 4, true, true>;
    if (variant == kVariantLdgPfU3) return (const void *)step_kernel_ldg<false, 3, true, true>;
    if (variant == kVariantLdgPfProducts) return (const void *)step_kernel_ldg<true, 3, false, true>;
    if (variant == kVariantPersist) return (const void *)step_kernel_persist<4>;
    if (variant == kVariantAsyncProducts) return (const void *)step_kernel_async<true, 3>;
    return (const void *)step_kernel_ldg<false, 1>;
}
}  // namespace

int step_kernel_prepare(int variant, size_t smem) {
    if (plain_loads(variant)) return 0;
    const void *k = kernel_of(variant);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return (int)e;
}

int step_kernel_occupancy(int variant, int block, size_t smem, int *blocks_per_sm) {
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel_of(variant), block,
                                                             plain_loads(variant) ? 0 : smem);
}

int step_kernel_attributes(int variant, int *regs, int *local_bytes) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel_of(variant));
    if (e != cudaSuccess) return (int)e;
    *regs = fa.numRegs;
    *local_bytes = (int)fa.localSizeBytes;
    return 0;
}

}  // namespace s2d

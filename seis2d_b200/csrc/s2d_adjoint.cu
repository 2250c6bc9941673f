// Adjoint FD step and gradient finalisation of libseis2d (sm_100a).
//
// The forward step (cpumodelling.cpp:115-156) written with its derivatives
//   a = Gx vx, c = Gz vz                      (D-, cpu_modelling_kernels.cpp:201-258)
//   px' = Dax px + Kx kappa a (+ source),  pz' = Daz pz + Kz kappa c
//   p' = px' + pz',  g = Hx p', h = Hz p'    (D+, :260-316)
//   vx' = Dbx vx + Lx bx g,  vz' = Dbz vz + Lz bz h
// is linear in the state.  One adjoint step maps the adjoint state after step
// kt, (mpx', mpz', mvx', mvz'), to the one before it:
//   mg = Lx bx mvx',  mh = Lz bz mvz'
//   q  = Hx^T mg + Hz^T mh (+ the adjoint source at the receivers)
//   mPX = mpx' + q,  mPZ = mpz' + q
//   mpx = Dax mPX,  mpz = Daz mPZ
//   mvx = Dbx mvx' + Gx^T (Kx kappa mPX),  mvz = Dbz mvz' + Gz^T (Kz kappa mPZ)
// and accumulates the imaging terms
//   dJ/dkappa += Kx a mPX + Kz c mPZ,  dJ/dbx += Lx g mvx',  dJ/dbz += Lz h mvz'
// with a, c, g, h of step kt saved by the forward (S2D_STEP_PRODUCTS); the
// last two go straight into dJ/db through the buoyancy averages.  All shots of
// a gradient call share one model, so they share one accumulator pair
// (dJ/dkappa, dJ/db): the terms are added with vector atomics (red.global
// .add.v4.f32), which keeps the pair in L2 instead of reading and writing a
// pair per shot from DRAM every step.  The order in which the shots' terms
// of one step arrive is not fixed, so gradients of several shots are
// reproducible to rounding, not bit for bit; one shot's are bit-exact.
//
// The transposes are the gather forms of the reference's operators, edge rows
// included: with (c0(j), c1(j)) the coefficient pair of forward row j,
//   (G^T m)[i] = c0(i) m[i] - c0(i+1) m[i+1] + c1(i-1) m[i-1] - c1(i+2) m[i+2]
//   (H^T m)[i] = c0(i-1) m[i-1] - c0(i) m[i] + c1(i-2) m[i-2] - c1(i+1) m[i+1]
// The kernel streams like the forward: a warp owns a 128-row strip, q and the
// pressure adjoint at column L-1, the velocity adjoint at column L-3.
#include <cuda_runtime.h>

#include "s2d_device.cuh"

namespace s2d {

namespace {

__device__ __forceinline__ float xc0m(int i, int n) { float c0, c1; dm_coef(i, n, c0, c1); return c0; }
__device__ __forceinline__ float xc1m(int i, int n) { float c0, c1; dm_coef(i, n, c0, c1); return c1; }
__device__ __forceinline__ float xc0p(int i, int n) { float c0, c1; dp_coef(i, n, c0, c1); return c0; }
__device__ __forceinline__ float xc1p(int i, int n) { float c0, c1; dp_coef(i, n, c0, c1); return c1; }


// (H^T m) at the lane's 4 rows from m at those rows and the neighbours' edge
// values (up_z = m[z0-2], up_w = m[z0-1], dn_x = m[z0+4]); pairs of rows z0-2 .. z0+4.
template <bool FAST>
__device__ __forceinline__ float4 hzt(const Lane<FAST> &ln, const float4 &m, float up_z, float up_w, float dn_x) {
    float a0, a1, b0, b1, c0, c1, d0, d1, e0, e1, f0, f1, g0, g1;
    zdp(ln, -2, a0, a1);
    zdp(ln, -1, b0, b1);
    zdp(ln, 0, c0, c1);
    zdp(ln, 1, d0, d1);
    zdp(ln, 2, e0, e1);
    zdp(ln, 3, f0, f1);
    zdp(ln, 4, g0, g1);
    float4 r;
    r.x = b0 * up_w - c0 * m.x + a1 * up_z - d1 * m.y;
    r.y = c0 * m.x - d0 * m.y + b1 * up_w - e1 * m.z;
    r.z = d0 * m.y - e0 * m.z + c1 * m.x - f1 * m.w;
    r.w = e0 * m.z - f0 * m.w + d1 * m.y - g1 * dn_x;
    return r;
}
// (G^T m) at the lane's 4 rows (up_w = m[z0-1], dn_x = m[z0+4], dn_y = m[z0+5]);
// pairs of rows z0-1 .. z0+5.
template <bool FAST>
__device__ __forceinline__ float4 gzt(const Lane<FAST> &ln, const float4 &m, float up_w, float dn_x, float dn_y) {
    float a0, a1, b0, b1, c0, c1, d0, d1, e0, e1, f0, f1, g0, g1;
    zdm(ln, -1, a0, a1);
    zdm(ln, 0, b0, b1);
    zdm(ln, 1, c0, c1);
    zdm(ln, 2, d0, d1);
    zdm(ln, 3, e0, e1);
    zdm(ln, 4, f0, f1);
    zdm(ln, 5, g0, g1);
    float4 r;
    r.x = b0 * m.x - c0 * m.y + a1 * up_w - d1 * m.z;
    r.y = c0 * m.y - d0 * m.z + b1 * m.x - e1 * m.w;
    r.z = d0 * m.z - e0 * m.w + c1 * m.y - f1 * dn_x;
    r.w = e0 * m.w - f0 * dn_x + d1 * m.z - g1 * dn_y;
    return r;
}

// One (shot, strip, segment) task of the adjoint step.  The warp streams
// along x: at column L it loads mvx' (the x-gather of H^T needs it at
// Q-2 .. Q+1); the pressure adjoint, the z-velocity adjoint and the imaging
// terms are formed at Q = L-1, the x-velocity adjoint at W = L-3 (its G^T
// x-gather needs Kx kappa mPX at W-1 .. W+2).
//
// Cells where both pressure dampings are 1 run the forward with p alone
// (p' = p + kappa (Kx a + Kz c)); their adjoint carries one pressure field
// (mpx, mpz unused) and the forward saved Kx a + Kz c in the first product
// slot.
//
// Imaging per step: dJ/dkappa += Kx a mPX + Kz c mPZ at Q.  The buoyancy
// terms tbx = Lx g mvx', tbz = Lz h mvz' enter dJ/db through the averages
// bx = (b[x] + b[x+1]) / 2, bz = (b[z] + b[z+1]) / 2 (cpu_modelling_kernels.cpp:89-119):
// dJ/db(Q, z) += (tbx(Q) + tbx(Q-1)) / 2 + (tbz(z) + tbz(z-1)) / 2.
// tbx at the last column and tbz at the last row vanish (the forward D+
// rows there are zero), so the reference's last-row / last-column
// replication adds nothing.  tbx(Q-1) comes from the previous column
// (computed at Q = xa-1 too), tbz(z-1) from the lane above.
// Per-warp shared-memory delay lines of the adjoint step (4 columns each):
// mvx', Lx bx mvx' and Kx kappa mPX, the inputs of its x-gathers.
constexpr int kAdjRing = 4, kAdjFields = 3;
constexpr int kAdjWarpBytes = kAdjRing * kAdjFields * S2D_STRIP_ROWS * 4;
__device__ __forceinline__ float4 &adj_ring(float4 *ring, int field, int col, int lane) {
    return ring[(field * kAdjRing + ((col + 2 * S2D_GX) & (kAdjRing - 1))) * 32 + lane];
}

// The loads of one column L of the adjoint loop (prefetching form): mvx'
// and bx at L; at Q = L-1 the column coefficients, mpx, mvz, mpz, bz, kappa
// and the step's products (first two slots where the lane updates Q, last two
// where Q is imaged).
struct AdjIn {
    float4 m, b, xq, mpx, mvz, mpz, bz, kk, pa, pc, pg, ph;
    float lx;
};

// Asynchronous form: the eleven column inputs of AdjIn (mvx', bx at L;
// mpx, mvz, mpz, bz, kappa and the four product slots at Q = L-1) as 16-byte
// cp.async copies into a per-warp ring of AS columns, issued AS-1 columns
// ahead, so the loads in flight hold no registers.  Each lane reads back only
// what it copied; inputs a column does not use are zero-filled copies that
// read nothing.
// With 3 or more columns in the ring the materials (bx, bz, kappa: shared by
// the shots, L2-resident) are loaded where they are used instead, and the ring
// holds the eight per-shot inputs, so three columns fit three blocks per SM.
__host__ __device__ constexpr int adj_async_slots(int as) { return as == 0 ? 0 : as < 3 ? 11 : 8; }
__host__ __device__ constexpr int adj_async_stage_bytes(int as) { return adj_async_slots(as) * S2D_STRIP_ROWS * 4; }

// XF: every column the task touches (xa-3 .. xb+2) lies in the shot's
// x-interior: literal column coefficients, no coefficient loads.  PF: the
// loads of column L+1 are issued before column L is computed (two columns
// in flight per warp); AS > 0: asynchronous copies AS-1 columns ahead into
// `aring`; otherwise each value is loaded where it is used.
template <bool FAST, bool XF = false, bool PF = false, int AS = 0>
__device__ __forceinline__ void adjoint_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len,
                                             int kt, int lane, float4 *ring, float4 *aring = nullptr) {
    const int nnx = S.nnx;
    const size_t ld = (size_t)S.ld;
    const int xb = min(nnx, xa + seg_len);
    const int c = strip * S2D_STRIP_OUT - 4;
    Lane<FAST> ln;
    lane_setup(ln, S, c, lane, kt);
    const int z0 = ln.z0;
    const int pin = (kt + 1) & 1, pout = kt & 1;
    const size_t off = (size_t)(ln.zl + S2D_GZ) + (size_t)S2D_GX * ld;
    const size_t F = (size_t)(nnx + 2 * S2D_GX) * ld;
    // Every buffer below is distinct: restrict lets the compiler issue the
    // accumulator and product loads ahead of the state stores.  (Per-field
    // pointers here: the base-and-stride form the forward kernels use costs
    // this kernel more address arithmetic than it saves in spills.)
    const float *__restrict__ mpxi = S.st[pin][0] + off;
    const float *__restrict__ mpzi = S.st[pin][1] + off;
    const float *__restrict__ mvxi = S.st[pin][2] + off;
    const float *__restrict__ mvzi = S.st[pin][3] + off;
    float *__restrict__ mpxo = S.st[pout][0] + off;
    float *__restrict__ mpzo = S.st[pout][1] + off;
    float *__restrict__ mvxo = S.st[pout][2] + off;
    float *__restrict__ mvzo = S.st[pout][3] + off;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = S.bx + off;
    const float *__restrict__ bzp = S.bz + off;
    const float *__restrict__ pr = S.prod + (size_t)(kt - a.prod_kt0) * 4 * F + off;
    float *__restrict__ gk = S.grad[0] + off;
    float *__restrict__ gb = S.grad[1] + off;
    // receiver adjoint source on recording steps, in strips whose rows hold
    // receivers (the lookup is three dependent loads per column)
    const bool inj = !(a.flags & S2D_STEP_NO_RECORD) && ((kt + 1) % a.dt_factor) == 0 &&
                     (kt + 1) / a.dt_factor - 1 < S.real_nt && c + S2D_STRIP_ROWS > S.rec_zlo &&
                     c <= S.rec_zhi;
    const int slot = (kt + 1) / a.dt_factor - 1;
    const bool row0 = FAST || z0 >= 1;  // the lane's first row has a row above it in the grid

    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 tbp = zero;                                      // tbx at Q-1
    const float kx = S.kx_in;
    auto fetch = [&](int L, AdjIn &in) {
        const ptrdiff_t colL = (ptrdiff_t)L * (ptrdiff_t)ld;
        in.m = ld4(mvxi + colL);
        in.b = ld4(bxp + colL);
        in.lx = XF ? kx : __ldg(S.xcoef + (L + S2D_GX)).w;
        if (L < xa) return;
        const int Q = L - 1;
        const ptrdiff_t colQ = (ptrdiff_t)Q * (ptrdiff_t)ld;
        in.xq = XF ? make_float4(1.0f, kx, 1.0f, kx) : __ldg(S.xcoef + (Q + S2D_GX));
        const bool pz_live = !(FAST && (XF || in.xq.x == 1.0f));
        const bool upd = Q >= xa && Q < xb && ln.owner;
        const bool img = Q >= 0 && Q < xb;
        in.mpx = ld4(mpxi + colQ);
        in.mvz = ld4(mvzi + colQ);
        in.mpz = pz_live ? ld4(mpzi + colQ) : zero;
        in.bz = ld4(bzp + colQ);
        in.kk = ld4(kap + colQ);
        in.pa = upd ? ld4(pr + colQ) : zero;
        in.pc = upd && pz_live ? ld4(pr + F + colQ) : zero;
        in.pg = img ? ld4(pr + 2 * F + colQ) : zero;
        in.ph = img ? ld4(pr + 3 * F + colQ) : zero;
    };
    AdjIn cur, nxt;
    if (PF) fetch(xa - 3, nxt);
    // asynchronous form: iteration i is column L = xa-3+i; ring slots
    // (times 32 float4) of its inputs
    constexpr bool kMatRing = AS < 3;
    constexpr int kSlots = adj_async_slots(AS);
    constexpr int sM = 0, sB = 1, sPX = kMatRing ? 2 : 1, sVZ = sPX + 1, sPZ = sPX + 2, sBZ = 5, sKK = 6;
    constexpr int sPA = kMatRing ? 7 : 4, sPC = sPA + 1, sPG = sPA + 2, sPH = sPA + 3;
    const int n_it = xb - xa + 6;
    auto issue = [&](int i) {
        float4 *st = aring + (i % (AS > 0 ? AS : 1)) * kSlots * 32 + lane;
        const int L = xa - 3 + i;
        const ptrdiff_t colL = (ptrdiff_t)L * (ptrdiff_t)ld;
        cp_async16(st + sM * 32, mvxi + colL, true);
        if (kMatRing) cp_async16(st + sB * 32, bxp + colL, true);
        if (L < xa) return;
        const int Q = L - 1;
        const ptrdiff_t colQ = (ptrdiff_t)Q * (ptrdiff_t)ld;
        const bool pz_live = !(FAST && (XF || __ldg(S.xcoef + (Q + S2D_GX)).x == 1.0f));
        const bool upd = Q >= xa && Q < xb && ln.owner;
        const bool img = Q >= 0 && Q < xb;
        cp_async16(st + sPX * 32, mpxi + colQ, true);
        cp_async16(st + sVZ * 32, mvzi + colQ, true);
        cp_async16(st + sPZ * 32, mpzi + colQ, pz_live);
        if (kMatRing) {
            cp_async16(st + sBZ * 32, bzp + colQ, true);
            cp_async16(st + sKK * 32, kap + colQ, true);
        }
        cp_async16(st + sPA * 32, pr + colQ, upd);
        cp_async16(st + sPC * 32, pr + F + colQ, upd && pz_live);
        cp_async16(st + sPG * 32, pr + 2 * F + colQ, img);
        cp_async16(st + sPH * 32, pr + 3 * F + colQ, img);
    };
    if constexpr (AS > 0) {
#pragma unroll
        for (int i = 0; i < AS - 1; ++i) {
            if (i < n_it) issue(i);
            cp_async_commit();
        }
    }
    const float4 *as = aring;  // this column's ring slots (asynchronous form)

    for (int L = xa - 3; L <= xb + 2; ++L) {
        if (PF) {
            cur = nxt;
            if (L < xb + 2) fetch(L + 1, nxt);
        }
        if constexpr (AS > 0) {
            const int i = L - (xa - 3);
            if (i + AS - 1 < n_it) issue(i + AS - 1);
            cp_async_commit();
            cp_async_wait<AS - 1>();  // column L's copies have landed
            as = aring + (i % AS) * kSlots * 32 + lane;
        }
        {
            const ptrdiff_t colL = (ptrdiff_t)L * (ptrdiff_t)ld;
            const float4 m = PF ? cur.m : AS ? as[sM * 32] : ld4(mvxi + colL);
            const float4 b = PF ? cur.b : AS && kMatRing ? as[sB * 32] : ld4(bxp + colL);
            const float lx = PF ? cur.lx : XF ? kx : __ldg(S.xcoef + (L + S2D_GX)).w;
            adj_ring(ring, 0, L, lane) = m;
            adj_ring(ring, 1, L, lane) = make_float4((lx * b.x) * m.x, (lx * b.y) * m.y, (lx * b.z) * m.z,
                                                     (lx * b.w) * m.w);
        }
        if (L < xa) continue;
        const int Q = L - 1;
        const ptrdiff_t colQ = (ptrdiff_t)Q * (ptrdiff_t)ld;
        const bool in_seg = Q >= xa && Q < xb;
        const bool upd = in_seg && ln.owner;       // this lane writes column Q
        const bool img = Q >= 0 && Q < xb;         // buoyancy terms at Q (xa-1 feeds column xa)
        const float4 xq = PF ? cur.xq : XF ? make_float4(1.0f, kx, 1.0f, kx) : __ldg(S.xcoef + (Q + S2D_GX));
        const bool colm = XF || xq.x == 1.0f;  // xq: Dax, Kx, Dbx, Lx at Q
        const bool pz_live = !(FAST && colm);  // some cell of the column keeps mpz
        const float4 mpx = PF ? cur.mpx : AS ? as[sPX * 32] : ld4(mpxi + colQ);
        const float4 mvz = PF ? cur.mvz : AS ? as[sVZ * 32] : ld4(mvzi + colQ);
        const float4 mpz = PF ? cur.mpz : AS ? as[sPZ * 32] : pz_live ? ld4(mpzi + colQ) : zero;
        const float4 bz = PF ? cur.bz : AS && kMatRing ? as[sBZ * 32] : ld4(bzp + colQ);
        const float4 kk = PF ? cur.kk : AS && kMatRing ? as[sKK * 32] : ld4(kap + colQ);
        float4 pa = zero, pc = zero, pg = zero, ph = zero, tk = zero, tb = zero;
        if (PF) {
            pa = cur.pa;
            pc = cur.pc;
            pg = cur.pg;
            ph = cur.ph;
        } else if (AS) {
            pa = as[sPA * 32];
            pc = as[sPC * 32];
            pg = as[sPG * 32];
            ph = as[sPH * 32];
        } else {
            if (upd) {
                pa = ld4(pr + colQ);
                if (pz_live) pc = ld4(pr + F + colQ);
            }
            if (img) {
                pg = ld4(pr + 2 * F + colQ);
                ph = ld4(pr + 3 * F + colQ);
            }
        }
        const float4 r0 = zrow(ln, 0), r1 = zrow(ln, 1), r2 = zrow(ln, 2), r3 = zrow(ln, 3);
        // merged cells (both pressure dampings 1) carry one pressure adjoint
        const bool m0 = colm && (FAST || r0.x == 1.0f), m1 = colm && (FAST || r1.x == 1.0f);
        const bool m2 = colm && (FAST || r2.x == 1.0f), m3 = colm && (FAST || r3.x == 1.0f);
        // ---- pressure adjoint at Q ----
        const float4 h = make_float4((r0.w * bz.x) * mvz.x, (r1.w * bz.y) * mvz.y, (r2.w * bz.z) * mvz.z,
                                     (r3.w * bz.w) * mvz.w);
        float4 q = hzt(ln, h, __shfl_up_sync(kFull, h.z, 1), __shfl_up_sync(kFull, h.w, 1),
                       __shfl_down_sync(kFull, h.x, 1));
        {
            const float p0a = XF ? kA0 : xc0p(Q - 1, nnx), p0b = XF ? kA0 : xc0p(Q, nnx);
            const float p1a = XF ? kA1 : xc1p(Q - 2, nnx), p1b = XF ? kA1 : xc1p(Q + 1, nnx);
            const float4 mg0 = adj_ring(ring, 1, L - 3, lane), mg1 = adj_ring(ring, 1, L - 2, lane);
            const float4 mg2 = adj_ring(ring, 1, L - 1, lane), mg3 = adj_ring(ring, 1, L, lane);
            q.x += p0a * mg1.x - p0b * mg2.x + p1a * mg0.x - p1b * mg3.x;
            q.y += p0a * mg1.y - p0b * mg2.y + p1a * mg0.y - p1b * mg3.y;
            q.z += p0a * mg1.z - p0b * mg2.z + p1a * mg0.z - p1b * mg3.z;
            q.w += p0a * mg1.w - p0b * mg2.w + p1a * mg0.w - p1b * mg3.w;
        }
        // Transpose of the receiver sampling (cpumodelling.cpp:356-360).  Every
        // warp computing column Q adds it (halo columns included, they feed the
        // neighbours' velocity adjoint); the receiver table covers columns
        // [0, nnx) only.
        if (inj && Q >= 0 && Q < nnx) {
            const int j1 = __ldg(S.rec_ptr + Q + 1);
            for (int j = __ldg(S.rec_ptr + Q); j < j1; ++j) {
                const int d = __ldg(S.rec_z + j) - z0;
                if (d >= 0 && d < 4) {
                    const float r = __ldg(S.seis + (size_t)__ldg(S.rec_id + j) * S.real_nt + slot);
                    if (d == 0) q.x += r;
                    else if (d == 1) q.y += r;
                    else if (d == 2) q.z += r;
                    else q.w += r;
                }
            }
        }
        const float4 mPX = make_float4(mpx.x + q.x, mpx.y + q.y, mpx.z + q.z, mpx.w + q.w);
        const float4 mPZ = make_float4(m0 ? mPX.x : mpz.x + q.x, m1 ? mPX.y : mpz.y + q.y,
                                       m2 ? mPX.z : mpz.z + q.z, m3 ? mPX.w : mpz.w + q.w);
        if (upd) {
            st4(mpxo + colQ, make_float4(xq.x * mPX.x, xq.x * mPX.y, xq.x * mPX.z, xq.x * mPX.w));
            if (pz_live)
                st4(mpzo + colQ, make_float4(m0 ? 0.0f : r0.x * mPZ.x, m1 ? 0.0f : r1.x * mPZ.y,
                                             m2 ? 0.0f : r2.x * mPZ.z, m3 ? 0.0f : r3.x * mPZ.w));
            // merged cells saved Kx a + Kz c in the first product slot
            tk.x += m0 ? pa.x * mPX.x : (xq.y * pa.x) * mPX.x + (r0.y * pc.x) * mPZ.x;
            tk.y += m1 ? pa.y * mPX.y : (xq.y * pa.y) * mPX.y + (r1.y * pc.y) * mPZ.y;
            tk.z += m2 ? pa.z * mPX.z : (xq.y * pa.z) * mPX.z + (r2.y * pc.z) * mPZ.z;
            tk.w += m3 ? pa.w * mPX.w : (xq.y * pa.w) * mPX.w + (r3.y * pc.w) * mPZ.w;
            red_add4(gk + colQ, tk);
            if (Q == S.src_x && ln.sdz >= 0 && ln.sdz < 4) S.srcadj[kt] = comp(mPX, ln.sdz);
        }
        adj_ring(ring, 2, Q, lane) = make_float4((xq.y * kk.x) * mPX.x, (xq.y * kk.y) * mPX.y, (xq.y * kk.z) * mPX.z,
                          (xq.y * kk.w) * mPX.w);
        // ---- z-velocity adjoint at Q ----
        {
            const float4 mc = make_float4((r0.y * kk.x) * mPZ.x, (r1.y * kk.y) * mPZ.y, (r2.y * kk.z) * mPZ.z,
                                          (r3.y * kk.w) * mPZ.w);
            const float4 g = gzt(ln, mc, __shfl_up_sync(kFull, mc.w, 1), __shfl_down_sync(kFull, mc.x, 1),
                                 __shfl_down_sync(kFull, mc.y, 1));
            if (upd)
                st4(mvzo + colQ, make_float4(r0.z * mvz.x + g.x, r1.z * mvz.y + g.y, r2.z * mvz.z + g.z,
                                             r3.z * mvz.w + g.w));
        }
        // ---- buoyancy imaging at Q ----
        if (img) {
            const float4 mv2 = adj_ring(ring, 0, Q, lane);
            const float4 tbx = make_float4((xq.w * pg.x) * mv2.x, (xq.w * pg.y) * mv2.y, (xq.w * pg.z) * mv2.z,
                                           (xq.w * pg.w) * mv2.w);
            const float4 tbz = make_float4((r0.w * ph.x) * mvz.x, (r1.w * ph.y) * mvz.y, (r2.w * ph.z) * mvz.z,
                                           (r3.w * ph.w) * mvz.w);
            const float up = __shfl_up_sync(kFull, tbz.w, 1);
            if (upd) {
                const float4 px = Q >= 1 ? tbp : zero;
                tb.x += 0.5f * ((tbx.x + px.x) + (tbz.x + (row0 ? up : 0.0f)));
                tb.y += 0.5f * ((tbx.y + px.y) + (tbz.y + tbz.x));
                tb.z += 0.5f * ((tbx.z + px.z) + (tbz.z + tbz.y));
                tb.w += 0.5f * ((tbx.w + px.w) + (tbz.w + tbz.z));
                red_add4(gb + colQ, tb);
            }
            tbp = tbx;
        }
        if (L < xa + 3) continue;
        // ---- x-velocity adjoint at W = L - 3 ----
        const int W = L - 3;
        const ptrdiff_t colW = (ptrdiff_t)W * (ptrdiff_t)ld;
        const float dbx = XF ? 1.0f : __ldg(S.xcoef + (W + S2D_GX)).z;
        const float m0a = XF ? kA0 : xc0m(W, nnx), m0b = XF ? kA0 : xc0m(W + 1, nnx);
        const float m1a = XF ? kA1 : xc1m(W - 1, nnx), m1b = XF ? kA1 : xc1m(W + 2, nnx);
        const float4 mv0 = adj_ring(ring, 0, W, lane);
        const float4 ma0 = adj_ring(ring, 2, W - 1, lane), ma1 = adj_ring(ring, 2, W, lane);
        const float4 ma2 = adj_ring(ring, 2, W + 1, lane), ma3 = adj_ring(ring, 2, W + 2, lane);
        float4 ovx;
        ovx.x = dbx * mv0.x + (m0a * ma1.x - m0b * ma2.x + m1a * ma0.x - m1b * ma3.x);
        ovx.y = dbx * mv0.y + (m0a * ma1.y - m0b * ma2.y + m1a * ma0.y - m1b * ma3.y);
        ovx.z = dbx * mv0.z + (m0a * ma1.z - m0b * ma2.z + m1a * ma0.z - m1b * ma3.z);
        ovx.w = dbx * mv0.w + (m0a * ma1.w - m0b * ma2.w + m1a * ma0.w - m1b * ma3.w);
        if (ln.owner) st4(mvxo + colW, ovx);
    }
    if constexpr (AS > 0) cp_async_wait<0>();
}

// MINB blocks of 4 warps per SM: 2 leaves the compiler its registers, 3 caps
// them at 168 (12 warps per SM), 4 at 128 (16 warps per SM, some spills).
// AS > 0: the asynchronous form with an AS-column copy ring per warp after
// its delay lines.
template <int MINB, bool PF = false, int AS = 0>
__global__ void __launch_bounds__(128, MINB) adjoint_kernel(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int kWarpBytes = kAdjWarpBytes + AS * adj_async_stage_bytes(AS);
    float4 *ring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kWarpBytes);
    float4 *aring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kWarpBytes + kAdjWarpBytes);
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base - kt_off;
    if (kt < 0 || kt >= a.fd_nt) return;
    // the task's shot record in this warp's shared-memory slot
    __shared__ ShotDev shot_rec[4];
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        if (!task_in_bounds(a, G, strip, xa, seg_len, kt, true, 2)) continue;
        warp_copy_shot(S, G, lane);
        const int c = strip * S2D_STRIP_OUT - 4;
        const int xb = min(S.nnx, xa + seg_len);
        // the z-transposes read the coefficient pairs of rows c-2 .. c+129,
        // the x-gathers those of columns xa-3 .. xb+2
        const bool zf = rows_fast(S, c - 2, c + S2D_STRIP_ROWS + 1);
        const bool xf = xa - 3 >= S.xfast_lo && xb + 2 < S.xfast_hi;
        if (zf && xf) adjoint_task<true, true, PF, AS>(a, S, strip, xa, seg_len, kt, lane, ring, aring);
        else if (zf) adjoint_task<true, false, PF, AS>(a, S, strip, xa, seg_len, kt, lane, ring, aring);
        else if (xf) adjoint_task<false, true, PF, AS>(a, S, strip, xa, seg_len, kt, lane, ring, aring);
        else adjoint_task<false, false, PF, AS>(a, S, strip, xa, seg_len, kt, lane, ring, aring);
    }
}

// ---- gradient finalisation ----

__device__ __forceinline__ size_t pad_id(int x, int z, int ld) {
    return (size_t)(x + S2D_GX) * ld + (z + S2D_GZ);
}

// Source term of dJ/dkappa (the amplitude fd_dt w kappa_src / (dx dz) depends
// on kappa at the source cell), added in shot order.
__global__ void add_source_terms(float *const *gk, const int *cells, const double *vals, int nshots) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int s = 0; s < nshots; ++s) gk[s][cells[s]] = (float)((double)gk[s][cells[s]] + vals[s]);
}

__global__ void sum_shots(float *const *gk, float *const *gb, int nshots, int nnx, int nnz, int ld, float *tk,
                          float *tb) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
    if (z >= nnz || x >= nnx) return;
    const size_t id = pad_id(x, z, ld);
    double a = 0, b = 0;
    for (int s = 0; s < nshots; ++s) {
        a += gk[s][id];
        b += gb[s][id];
    }
    tk[id] = (float)a;
    tb[id] = (float)b;
}

// kappa = vp^2 rho and b = 1/rho (the buoyancy averages are folded into dJ/db
// by the adjoint step).  Rows z < kfix hold kappa at 0 (free surface): their
// dJ/dkappa does not depend on vp or rho.
__global__ void chain_rule(const float *tk, const float *tb, const float *vp, const float *rho, int nx, int nz,
                           int nb, int ld, int kfix, float *gvp, float *grho) {
    const int nnx = nx + 2 * nb, nnz = nz + 2 * nb;
    const int z = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
    if (z >= nnz || x >= nnx) return;
    const size_t id = pad_id(x, z, ld);
    const double gb = tb[id];
    const double gk = z < kfix ? 0.0 : (double)tk[id];
    const int mx = min(max(x - nb, 0), nx - 1), mz = min(max(z - nb, 0), nz - 1);
    const double v = vp[(size_t)mx * nz + mz], r = rho[(size_t)mx * nz + mz];
    gvp[id] = (float)(2.0 * v * r * gk);
    grho[id] = (float)(v * v * gk + (r > 0 ? -gb / (r * r) : 0.0));
}

// Fold the sponge onto the model cells it replicates (transpose of
// cpumodelling.cpp:39-60).
__global__ void fold_sponge(const float *gvp, const float *grho, int nx, int nz, int nb, int ld, float *out_vp,
                            float *out_rho) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
    if (iz >= nz || ix >= nx) return;
    const int nnx = nx + 2 * nb, nnz = nz + 2 * nb;
    const int x0 = ix == 0 ? 0 : ix + nb, x1 = ix == nx - 1 ? nnx - 1 : ix + nb;
    const int z0 = iz == 0 ? 0 : iz + nb, z1 = iz == nz - 1 ? nnz - 1 : iz + nb;
    double a = 0, b = 0;
    for (int x = x0; x <= x1; ++x)
        for (int z = z0; z <= z1; ++z) {
            const size_t id = pad_id(x, z, ld);
            a += gvp[id];
            b += grho[id];
        }
    out_vp[(size_t)ix * nz + iz] = (float)a;
    out_rho[(size_t)ix * nz + iz] = (float)b;
}

__global__ void residual_kernel(const float *seis, const float *obs, float *res, size_t n, double *sumsq) {
    __shared__ double part[256];
#ifdef S2D_DEVICE_CHECKS
    if (blockDim.x != 256) return;
#endif
    double acc = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float r = seis[i] - obs[i];
        res[i] = r;
        acc += (double)r * r;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(sumsq, part[0]);
}

// ---------------------------------------------------------------- 8th order
//
// Adjoint step of the 8th-order scheme: the algebra of the header above with
// the 8-tap operators, in two cell-parallel passes (one thread per padded
// cell, blockIdx.z = shot; the gathers read their neighbours from memory):
//   pass 1: q = Hx^T(Lx bx mvx') + Hz^T(Lz bz mvz') (+ the adjoint source),
//           mPX, mPZ, the new mpx, mpz, dJ/dkappa, and Kx kappa mPX,
//           Kz kappa mPZ into the shot's two scratch fields;
//   pass 2: mvx = Dbx mvx' + Gx^T(Kx kappa mPX), mvz likewise, and dJ/db.
// Gather forms of the transposes, with c(j) the coefficients of forward row j
// (dm8 / dp8, zero outside the grid):
//   (G^T m)[i] = sum_k c_k(i-k) m[i-k] - c_k(i+1+k) m[i+1+k]
//   (H^T m)[i] = sum_k c_k(i-1-k) m[i-1-k] - c_k(i+k) m[i+k]
// (for the 4th-order pairs these are the gathers of adjoint_task).  The taps
// reach 4 cells, inside the 8 ghost columns and rows, whose scratch stays 0.

__device__ __forceinline__ size_t cell8(int x, int z, int ld) {
    return (size_t)(x + S2D_GX) * (size_t)ld + (size_t)(z + S2D_GZ);
}

__global__ void __launch_bounds__(128) adjoint8_pressure(const StepArgs *__restrict__ A, int kt_off) {
    const StepArgs a = *A;
    const int kt = a.kt_base - kt_off;
    if (kt < 0 || kt >= a.fd_nt) return;
    const ShotDev &S = a.shots[blockIdx.z];
    const int z = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
    if (z >= S.nnz || x >= S.nnx) return;
    const int ld = S.ld, nnx = S.nnx, nnz = S.nnz;
    const int pin = (kt + 1) & 1, pout = kt & 1;
    const size_t id = cell8(x, z, ld);
    const size_t F = (size_t)(nnx + 2 * S2D_GX) * (size_t)ld;
    const float *__restrict__ mvx = S.st[pin][2];
    const float *__restrict__ mvz = S.st[pin][3];
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j0 = x - 1 - k, j1 = x + k;
        const size_t i0 = cell8(j0, z, ld), i1 = cell8(j1, z, ld);
        q += comp(dp8(j0, nnx), k) * ((__ldg(S.xcoef + (j0 + S2D_GX)).w * __ldg(S.bx + i0)) * __ldg(mvx + i0));
        q -= comp(dp8(j1, nnx), k) * ((__ldg(S.xcoef + (j1 + S2D_GX)).w * __ldg(S.bx + i1)) * __ldg(mvx + i1));
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j0 = z - 1 - k, j1 = z + k;
        const size_t i0 = cell8(x, j0, ld), i1 = cell8(x, j1, ld);
        q += comp(dp8(j0, nnz), k) * ((__ldg(S.zcoef + (j0 + S2D_GZ)).w * __ldg(S.bz + i0)) * __ldg(mvz + i0));
        q -= comp(dp8(j1, nnz), k) * ((__ldg(S.zcoef + (j1 + S2D_GZ)).w * __ldg(S.bz + i1)) * __ldg(mvz + i1));
    }
    // transpose of the receiver sampling (cpumodelling.cpp:356-360)
    const int slot = (kt + 1) / a.dt_factor - 1;
    if (!(a.flags & S2D_STEP_NO_RECORD) && ((kt + 1) % a.dt_factor) == 0 && slot < S.real_nt) {
        const int j1 = __ldg(S.rec_ptr + x + 1);
        for (int j = __ldg(S.rec_ptr + x); j < j1; ++j)
            if (__ldg(S.rec_z + j) == z) q += __ldg(S.seis + (size_t)__ldg(S.rec_id + j) * S.real_nt + slot);
    }
    const float4 xq = __ldg(S.xcoef + (x + S2D_GX));  // Dax, Kx, Dbx, Lx
    const float4 r = __ldg(S.zcoef + (z + S2D_GZ));   // Daz, Kz, Dbz, Lz
    const bool merged = xq.x == 1.0f && r.x == 1.0f;   // the forward carried p alone here
    const float mPX = S.st[pin][0][id] + q;
    const float mPZ = merged ? mPX : S.st[pin][1][id] + q;
    S.st[pout][0][id] = xq.x * mPX;
    S.st[pout][1][id] = merged ? 0.0f : r.x * mPZ;
    const float *__restrict__ pr = S.prod + (size_t)(kt - a.prod_kt0) * 4 * F;
    const float pa = __ldg(pr + id);
    atomicAdd(S.grad[0] + id, merged ? pa * mPX : (xq.y * pa) * mPX + (r.y * __ldg(pr + F + id)) * mPZ);
    const float k = __ldg(S.kappa + id);
    S.scr[id] = (xq.y * k) * mPX;
    S.scr[F + id] = (r.y * k) * mPZ;
    if (x == S.src_x && z == S.src_z) S.srcadj[kt] = mPX;
}

__global__ void __launch_bounds__(128) adjoint8_velocity(const StepArgs *__restrict__ A, int kt_off) {
    const StepArgs a = *A;
    const int kt = a.kt_base - kt_off;
    if (kt < 0 || kt >= a.fd_nt) return;
    const ShotDev &S = a.shots[blockIdx.z];
    const int z = blockIdx.x * blockDim.x + threadIdx.x, x = blockIdx.y;
    if (z >= S.nnz || x >= S.nnx) return;
    const int ld = S.ld, nnx = S.nnx, nnz = S.nnz;
    const int pin = (kt + 1) & 1, pout = kt & 1;
    const size_t id = cell8(x, z, ld);
    const size_t F = (size_t)(nnx + 2 * S2D_GX) * (size_t)ld;
    const float *__restrict__ sa = S.scr;
    const float *__restrict__ sb = S.scr + F;
    float gx = 0.0f, gz = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx += comp(dm8(x - k, nnx), k) * __ldg(sa + cell8(x - k, z, ld));
        gx -= comp(dm8(x + 1 + k, nnx), k) * __ldg(sa + cell8(x + 1 + k, z, ld));
        gz += comp(dm8(z - k, nnz), k) * __ldg(sb + cell8(x, z - k, ld));
        gz -= comp(dm8(z + 1 + k, nnz), k) * __ldg(sb + cell8(x, z + 1 + k, ld));
    }
    const float4 xq = __ldg(S.xcoef + (x + S2D_GX));
    const float4 r = __ldg(S.zcoef + (z + S2D_GZ));
    const float *__restrict__ mvx = S.st[pin][2];
    const float *__restrict__ mvz = S.st[pin][3];
    const float vx_in = __ldg(mvx + id), vz_in = __ldg(mvz + id);
    S.st[pout][2][id] = xq.z * vx_in + gx;
    S.st[pout][3][id] = r.z * vz_in + gz;
    // buoyancy imaging: tbx = Lx g mvx', tbz = Lz h mvz' through the averages
    // bx = (b[x] + b[x+1]) / 2, bz = (b[z] + b[z+1]) / 2
    const float *__restrict__ pr = S.prod + (size_t)(kt - a.prod_kt0) * 4 * F;
    const float tbx = (xq.w * __ldg(pr + 2 * F + id)) * vx_in;
    const float tbz = (r.w * __ldg(pr + 3 * F + id)) * vz_in;
    const float tbxm = x >= 1 ? (__ldg(S.xcoef + (x - 1 + S2D_GX)).w * __ldg(pr + 2 * F + id - ld)) * __ldg(mvx + id - ld)
                              : 0.0f;
    const float tbzm = z >= 1 ? (__ldg(S.zcoef + (z - 1 + S2D_GZ)).w * __ldg(pr + 3 * F + id - 1)) * __ldg(mvz + id - 1)
                              : 0.0f;
    atomicAdd(S.grad[1] + id, 0.5f * ((tbx + tbxm) + (tbz + tbzm)));
}

// ---------------------------------------------------------------- 8th order, streaming
//
// The adjoint step of the 8th-order scheme as one streaming pass (the
// algebra of adjoint8_pressure / adjoint8_velocity, the same products in the
// same order per cell): a warp owns a 128-row strip read from 112k - 8 and
// writes its middle 112 rows (lanes 2..29, the 8th-order forward's layout),
// streaming along x.  At loop column L it loads mvx' and bx; at Q = L-3 it
// forms the pressure adjoint (x-gather of Lx bx mvx' over Q-4 .. Q+3, z-gather
// of Lz bz mvz' over the rows z-4 .. z+3 by shuffles from the neighbouring
// lanes), the z-velocity adjoint (z-gather of Kz kappa mPZ) and the imaging
// terms; at W = L-7 the x-velocity adjoint (x-gather of Kx kappa mPX over
// W-3 .. W+4).  The x-gathers read 8-column per-warp shared-memory rings of
// mvx', Lx bx mvx' and Kx kappa mPX; each lane reads back only what it wrote.
constexpr int kAdj8Ring = 8, kAdj8Fields = 3;
constexpr int kAdj8WarpBytes = kAdj8Ring * kAdj8Fields * S2D_STRIP_ROWS * 4;
__device__ __forceinline__ float4 &adj8_ring(float4 *ring, int field, int col, int lane) {
    return ring[(field * kAdj8Ring + ((col + 2 * S2D_GX) & (kAdj8Ring - 1))) * 32 + lane];
}
__device__ __forceinline__ float c8(const float4 &c, int k) { return comp(c, k); }

// FAST: every row the task touches is in the 8th-order z-interior (literal
// coefficients, no z-damping); XF: likewise every column.
template <bool FAST, bool XF>
__device__ __forceinline__ void adjoint8s_task(const StepArgs &a, const ShotDev &S, int strip, int xa, int seg_len,
                                               int kt, int lane, float4 *ring) {
    const int nnx = S.nnx, nnz = S.nnz;
    const size_t ld = (size_t)S.ld;
    const int xb = min(nnx, xa + seg_len);
    const int c = strip * S2D_TS_OUT - 8;
    const int z0 = c + S2D_ZPT * lane;
    const bool ghost = z0 < 0 || z0 >= nnz;
    const bool owner = lane >= 2 && lane <= 29 && !ghost;
    const int zl = ghost ? -S2D_GZ : z0;
    const int pin = (kt + 1) & 1, pout = kt & 1;
    const size_t off = (size_t)(zl + S2D_GZ) + (size_t)S2D_GX * ld;
    const size_t F = (size_t)(nnx + 2 * S2D_GX) * ld;
    const float *__restrict__ mpxi = S.st[pin][0] + off;
    const float *__restrict__ mpzi = S.st[pin][1] + off;
    const float *__restrict__ mvxi = S.st[pin][2] + off;
    const float *__restrict__ mvzi = S.st[pin][3] + off;
    float *__restrict__ mpxo = S.st[pout][0] + off;
    float *__restrict__ mpzo = S.st[pout][1] + off;
    float *__restrict__ mvxo = S.st[pout][2] + off;
    float *__restrict__ mvzo = S.st[pout][3] + off;
    const float *__restrict__ kap = S.kappa + off;
    const float *__restrict__ bxp = S.bx + off;
    const float *__restrict__ bzp = S.bz + off;
    const float *__restrict__ pr = S.prod + (size_t)(kt - a.prod_kt0) * 4 * F + off;
    float *__restrict__ gk = S.grad[0] + off;
    float *__restrict__ gb = S.grad[1] + off;
    // receiver adjoint source on recording steps, in strips whose rows hold
    // receivers (the lookup is three dependent loads per column)
    const bool inj = !(a.flags & S2D_STEP_NO_RECORD) && ((kt + 1) % a.dt_factor) == 0 &&
                     (kt + 1) / a.dt_factor - 1 < S.real_nt && c + S2D_STRIP_ROWS > S.rec_zlo &&
                     c <= S.rec_zhi;
    const int slot = (kt + 1) / a.dt_factor - 1;
    const float kx = S.kx_in, kz = S.kz_in;
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 lit = make_float4(kC81, kC82, kC83, kC84);
    // coefficient k of the forward D+ / D- row j (x: columns, z: rows)
    auto cpx = [&](int j, int k) { return XF ? comp(lit, k) : c8(dp8(j, nnx), k); };
    auto cmx = [&](int j, int k) { return XF ? comp(lit, k) : c8(dm8(j, nnx), k); };
    auto cpz = [&](int j, int k) { return FAST ? comp(lit, k) : c8(dp8(j, nnz), k); };
    auto cmz = [&](int j, int k) { return FAST ? comp(lit, k) : c8(dm8(j, nnz), k); };
    // z-row coefficients (Daz, Kz, Dbz, Lz) of the lane's row z0 + i
    auto zr = [&](int i) { return FAST ? make_float4(1.0f, kz, 1.0f, kz) : __ldg(S.zcoef + (z0 + i + S2D_GZ)); };
    float4 tbp = zero;  // tbx at Q-1
    for (int L = xa - 7; L <= xb + 6; ++L) {
        {
            const ptrdiff_t colL = (ptrdiff_t)L * (ptrdiff_t)ld;
            const float4 m = ld4(mvxi + colL), b = ld4(bxp + colL);
            const float lx = XF ? kx : __ldg(S.xcoef + (L + S2D_GX)).w;
            adj8_ring(ring, 0, L, lane) = m;
            adj8_ring(ring, 1, L, lane) = make_float4((lx * b.x) * m.x, (lx * b.y) * m.y, (lx * b.z) * m.z,
                                                      (lx * b.w) * m.w);
        }
        const int Q = L - 3;
        if (Q < xa - 3) continue;
        const ptrdiff_t colQ = (ptrdiff_t)Q * (ptrdiff_t)ld;
        const bool upd = owner && Q >= xa && Q < xb;
        const bool img = Q >= xa - 1 && Q < xb && Q >= 0;
        const float4 xq = XF ? make_float4(1.0f, kx, 1.0f, kx) : __ldg(S.xcoef + (Q + S2D_GX));
        const bool colm = XF || xq.x == 1.0f;
        const bool pz_live = !(FAST && colm);
        const float4 mvz = ld4(mvzi + colQ), bz = ld4(bzp + colQ), kk = ld4(kap + colQ);
        const float4 mpx = ld4(mpxi + colQ);
        const float4 mpz = pz_live ? ld4(mpzi + colQ) : zero;
        const float4 r0 = zr(0), r1 = zr(1), r2 = zr(2), r3 = zr(3);
        const bool m0 = colm && r0.x == 1.0f, m1 = colm && r1.x == 1.0f;
        const bool m2 = colm && r2.x == 1.0f, m3 = colm && r3.x == 1.0f;
        // ---- pressure adjoint at Q ----
        float qv[4];
        {
            // x-gather of g = Lx bx mvx' (columns Q-4 .. Q+3 in ring 1)
            float4 acc = zero;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int j0 = Q - 1 - k, j1 = Q + k;
                const float c0 = cpx(j0, k), c1 = cpx(j1, k);
                const float4 g0 = adj8_ring(ring, 1, j0, lane), g1 = adj8_ring(ring, 1, j1, lane);
                acc.x += c0 * g0.x; acc.x -= c1 * g1.x;
                acc.y += c0 * g0.y; acc.y -= c1 * g1.y;
                acc.z += c0 * g0.z; acc.z -= c1 * g1.z;
                acc.w += c0 * g0.w; acc.w -= c1 * g1.w;
            }
            // z-gather of h = Lz bz mvz' over rows z-4 .. z+3: rows z0-4 .. z0+6
            const float4 h = make_float4((r0.w * bz.x) * mvz.x, (r1.w * bz.y) * mvz.y, (r2.w * bz.z) * mvz.z,
                                         (r3.w * bz.w) * mvz.w);
            float hh[11];
            hh[0] = __shfl_up_sync(kFull, h.x, 1);
            hh[1] = __shfl_up_sync(kFull, h.y, 1);
            hh[2] = __shfl_up_sync(kFull, h.z, 1);
            hh[3] = __shfl_up_sync(kFull, h.w, 1);
            hh[4] = h.x; hh[5] = h.y; hh[6] = h.z; hh[7] = h.w;
            hh[8] = __shfl_down_sync(kFull, h.x, 1);
            hh[9] = __shfl_down_sync(kFull, h.y, 1);
            hh[10] = __shfl_down_sync(kFull, h.z, 1);
            qv[0] = acc.x; qv[1] = acc.y; qv[2] = acc.z; qv[3] = acc.w;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int z = z0 + i;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    qv[i] += cpz(z - 1 - k, k) * hh[4 + i - 1 - k];
                    qv[i] -= cpz(z + k, k) * hh[4 + i + k];
                }
            }
        }
        // transpose of the receiver sampling (cpumodelling.cpp:356-360)
        if (inj && Q >= 0 && Q < nnx) {
            const int j1 = __ldg(S.rec_ptr + Q + 1);
            for (int j = __ldg(S.rec_ptr + Q); j < j1; ++j) {
                const int d = __ldg(S.rec_z + j) - z0;
                if (d >= 0 && d < 4) qv[d] += __ldg(S.seis + (size_t)__ldg(S.rec_id + j) * S.real_nt + slot);
            }
        }
        const float4 mPX = make_float4(mpx.x + qv[0], mpx.y + qv[1], mpx.z + qv[2], mpx.w + qv[3]);
        const float4 mPZ = make_float4(m0 ? mPX.x : mpz.x + qv[0], m1 ? mPX.y : mpz.y + qv[1],
                                       m2 ? mPX.z : mpz.z + qv[2], m3 ? mPX.w : mpz.w + qv[3]);
        if (upd) {
            st4(mpxo + colQ, make_float4(xq.x * mPX.x, xq.x * mPX.y, xq.x * mPX.z, xq.x * mPX.w));
            if (pz_live)
                st4(mpzo + colQ, make_float4(m0 ? 0.0f : r0.x * mPZ.x, m1 ? 0.0f : r1.x * mPZ.y,
                                             m2 ? 0.0f : r2.x * mPZ.z, m3 ? 0.0f : r3.x * mPZ.w));
            const float4 pa = ld4(pr + colQ);
            const float4 pc = pz_live ? ld4(pr + F + colQ) : zero;
            float4 tk;
            tk.x = m0 ? pa.x * mPX.x : (xq.y * pa.x) * mPX.x + (r0.y * pc.x) * mPZ.x;
            tk.y = m1 ? pa.y * mPX.y : (xq.y * pa.y) * mPX.y + (r1.y * pc.y) * mPZ.y;
            tk.z = m2 ? pa.z * mPX.z : (xq.y * pa.z) * mPX.z + (r2.y * pc.z) * mPZ.z;
            tk.w = m3 ? pa.w * mPX.w : (xq.y * pa.w) * mPX.w + (r3.y * pc.w) * mPZ.w;
            red_add4(gk + colQ, tk);
            if (Q == S.src_x && S.src_z - z0 >= 0 && S.src_z - z0 < 4) S.srcadj[kt] = comp(mPX, S.src_z - z0);
        }
        adj8_ring(ring, 2, Q, lane) = make_float4((xq.y * kk.x) * mPX.x, (xq.y * kk.y) * mPX.y,
                                                  (xq.y * kk.z) * mPX.z, (xq.y * kk.w) * mPX.w);
        // ---- z-velocity adjoint at Q: z-gather of sb = Kz kappa mPZ over rows z-3 .. z+4 ----
        {
            const float4 sb = make_float4((r0.y * kk.x) * mPZ.x, (r1.y * kk.y) * mPZ.y, (r2.y * kk.z) * mPZ.z,
                                          (r3.y * kk.w) * mPZ.w);
            float ss[11];  // rows z0-3 .. z0+7
            ss[0] = __shfl_up_sync(kFull, sb.y, 1);
            ss[1] = __shfl_up_sync(kFull, sb.z, 1);
            ss[2] = __shfl_up_sync(kFull, sb.w, 1);
            ss[3] = sb.x; ss[4] = sb.y; ss[5] = sb.z; ss[6] = sb.w;
            ss[7] = __shfl_down_sync(kFull, sb.x, 1);
            ss[8] = __shfl_down_sync(kFull, sb.y, 1);
            ss[9] = __shfl_down_sync(kFull, sb.z, 1);
            ss[10] = __shfl_down_sync(kFull, sb.w, 1);
            float gz[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int z = z0 + i;
                gz[i] = 0.0f;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    gz[i] += cmz(z - k, k) * ss[3 + i - k];
                    gz[i] -= cmz(z + 1 + k, k) * ss[3 + i + 1 + k];
                }
            }
            if (upd)
                st4(mvzo + colQ, make_float4(r0.z * mvz.x + gz[0], r1.z * mvz.y + gz[1], r2.z * mvz.z + gz[2],
                                             r3.z * mvz.w + gz[3]));
        }
        // ---- buoyancy imaging at Q ----
        if (img) {
            const float4 pg = ld4(pr + 2 * F + colQ);
            const float4 mv2 = adj8_ring(ring, 0, Q, lane);
            const float4 tbx = make_float4((xq.w * pg.x) * mv2.x, (xq.w * pg.y) * mv2.y, (xq.w * pg.z) * mv2.z,
                                           (xq.w * pg.w) * mv2.w);
            const float4 ph = ld4(pr + 3 * F + colQ);
            const float4 tbz = make_float4((r0.w * ph.x) * mvz.x, (r1.w * ph.y) * mvz.y, (r2.w * ph.z) * mvz.z,
                                           (r3.w * ph.w) * mvz.w);
            const float up = __shfl_up_sync(kFull, tbz.w, 1);  // img is the same for the whole warp
            if (upd) {
                const float4 px = Q >= 1 ? tbp : zero;
                float4 tb;
                tb.x = 0.5f * ((tbx.x + px.x) + (tbz.x + (z0 >= 1 ? up : 0.0f)));
                tb.y = 0.5f * ((tbx.y + px.y) + (tbz.y + tbz.x));
                tb.z = 0.5f * ((tbx.z + px.z) + (tbz.z + tbz.y));
                tb.w = 0.5f * ((tbx.w + px.w) + (tbz.w + tbz.z));
                red_add4(gb + colQ, tb);
            }
            tbp = tbx;
        }
        // ---- x-velocity adjoint at W = L - 7: x-gather of Kx kappa mPX over W-3 .. W+4 ----
        const int W = L - 7;
        if (W < xa || W >= xb || !owner) continue;
        const ptrdiff_t colW = (ptrdiff_t)W * (ptrdiff_t)ld;
        const float dbx = XF ? 1.0f : __ldg(S.xcoef + (W + S2D_GX)).z;
        const float4 mv0 = adj8_ring(ring, 0, W, lane);
        float4 gx = zero;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float c0 = cmx(W - k, k), c1 = cmx(W + 1 + k, k);
            const float4 s0 = adj8_ring(ring, 2, W - k, lane), s1 = adj8_ring(ring, 2, W + 1 + k, lane);
            gx.x += c0 * s0.x; gx.x -= c1 * s1.x;
            gx.y += c0 * s0.y; gx.y -= c1 * s1.y;
            gx.z += c0 * s0.z; gx.z -= c1 * s1.z;
            gx.w += c0 * s0.w; gx.w -= c1 * s1.w;
        }
        st4(mvxo + colW, make_float4(dbx * mv0.x + gx.x, dbx * mv0.y + gx.y, dbx * mv0.z + gx.z, dbx * mv0.w + gx.w));
    }
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) adjoint8s_kernel(const StepArgs *__restrict__ A, int kt_off) {
    extern __shared__ __align__(128) unsigned char smem[];
    float4 *ring = reinterpret_cast<float4 *>(smem + (size_t)(threadIdx.x >> 5) * kAdj8WarpBytes);
    const StepArgs a = *A;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * blockDim.x) >> 5);
    const int kt = a.kt_base - kt_off;
    if (kt < 0 || kt >= a.fd_nt) return;
    __shared__ ShotDev shot_rec[4];  // the task's shot record, one slot per warp
    ShotDev &S = shot_rec[(threadIdx.x >> 5) & 3];
    for (int t = gwarp; t < a.total_tasks; t += nwarp) {
        int strip, xa, seg_len;
        const ShotDev &G = task_of(a, t, strip, xa, seg_len);
        warp_copy_shot(S, G, lane);
        const int c = strip * S2D_TS_OUT - 8;
        const int xb = min(S.nnx, xa + seg_len);
        // rows c-4 .. c+131 take part (gathers reach 4 rows past the strip)
        const bool zf = rows_fast(S, c - 4, c + S2D_STRIP_ROWS + 3) && c - 4 >= 4 &&
                        c + S2D_STRIP_ROWS + 3 <= S.nnz - 5;
        // columns xa-7 .. xb+6 take part
        const bool xf = xa - 7 >= max(S.xfast_lo, 4) && xb + 6 < min(S.xfast_hi, S.nnx - 4);
        if (zf && xf) adjoint8s_task<true, true>(a, S, strip, xa, seg_len, kt, lane, ring);
        else if (zf) adjoint8s_task<true, false>(a, S, strip, xa, seg_len, kt, lane, ring);
        else if (xf) adjoint8s_task<false, true>(a, S, strip, xa, seg_len, kt, lane, ring);
        else adjoint8s_task<false, false>(a, S, strip, xa, seg_len, kt, lane, ring);
    }
}

}  // namespace

int launch_adjoint8s(const StepArgs *args_dev, int kt_off, int grid, void *stream) {
    adjoint8s_kernel<3><<<grid, 128, 4 * kAdj8WarpBytes, (cudaStream_t)stream>>>(args_dev, kt_off);
    return (int)cudaGetLastError();
}

// Also raises the kernel's dynamic shared-memory limit (its 48 KB of rings
// and the static shot records exceed the default); called before the
// launches.
int adjoint8s_occupancy(int *blocks_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(adjoint8s_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         4 * kAdj8WarpBytes);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, adjoint8s_kernel<3>, 128,
                                                             4 * kAdj8WarpBytes);
}

int launch_adjoint8(const StepArgs *args_dev, int kt_off, int nnx, int nnz, int nshots, void *stream) {
    const dim3 blk(128), grd((nnz + 127) / 128, nnx, nshots);
    adjoint8_pressure<<<grd, blk, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    adjoint8_velocity<<<grd, blk, 0, (cudaStream_t)stream>>>(args_dev, kt_off);
    return (int)cudaGetLastError();
}

namespace {
// minb 2, 3, 4: blocks per SM the kernel is built for; 12: 2 blocks per SM
// with the next column's loads prefetched
using AdjKernel = void (*)(const StepArgs *, int);
// Kernel of an `adjoint_blocks` code: 2, 3, 4 blocks per SM; 12: 2 with the
// register prefetch; 13: 3 with a 2-column copy ring; 14: 2 with a 3-column
// ring; 15: 3 with a 3-column ring of the per-shot inputs.
AdjKernel adjoint_kernel_of(int minb) {
    if (minb == 12) return adjoint_kernel<2, true>;
    if (minb == 13) return adjoint_kernel<3, false, 2>;
    if (minb == 14) return adjoint_kernel<2, false, 3>;
    if (minb == 15) return adjoint_kernel<3, false, 3>;
    return minb >= 4 ? adjoint_kernel<4> : minb == 3 ? adjoint_kernel<3> : adjoint_kernel<2>;
}
size_t adjoint_warp_bytes(int minb) {
    const int as = minb == 13 ? 2 : minb == 14 || minb == 15 ? 3 : 0;
    return (size_t)kAdjWarpBytes + (size_t)as * adj_async_stage_bytes(as);
}
}  // namespace

int launch_adjoint(const StepArgs *args_dev, int kt_off, int grid, int block, int minb, void *stream) {
    const size_t smem = (size_t)(block / 32) * adjoint_warp_bytes(minb);
    adjoint_kernel_of(minb)<<<grid, block, smem, (cudaStream_t)stream>>>(args_dev, kt_off);
    return (int)cudaGetLastError();
}

// Also raises the kernel's dynamic shared-memory limit (the copy-ring forms
// take more than 48 KB per block); called before the adjoint's launches.
int adjoint_kernel_occupancy(int block, int minb, int *blocks_per_sm) {
    const size_t smem = (size_t)(block / 32) * adjoint_warp_bytes(minb);
    cudaError_t e = cudaFuncSetAttribute(adjoint_kernel_of(minb), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, adjoint_kernel_of(minb), block, smem);
}

int launch_gradient_finalize(float *const *gk, float *const *gb, int nshots, int nacc, const int *src_cells,
                             const double *src_vals, const float *vp, const float *rho, int nx, int nz, int nb,
                             int ld, int kappa_fixed_rows, float *tmp2, float *gvp_pad, float *grho_pad,
                             float *grad_vp, float *grad_rho, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const int nnx = nx + 2 * nb, nnz = nz + 2 * nb;
    const size_t F = (size_t)(nnx + 2 * S2D_GX) * ld;
    add_source_terms<<<1, 1, 0, st>>>(gk, src_cells, src_vals, nshots);
    dim3 blk(256), grd((nnz + 255) / 256, nnx);
    sum_shots<<<grd, blk, 0, st>>>(gk, gb, nacc, nnx, nnz, ld, tmp2, tmp2 + F);
    chain_rule<<<grd, blk, 0, st>>>(tmp2, tmp2 + F, vp, rho, nx, nz, nb, ld, kappa_fixed_rows, gvp_pad, grho_pad);
    dim3 grd2((nz + 255) / 256, nx);
    fold_sponge<<<grd2, blk, 0, st>>>(gvp_pad, grho_pad, nx, nz, nb, ld, grad_vp, grad_rho);
    return (int)cudaGetLastError();
}

int launch_residual(const float *seis, const float *obs, float *res, size_t n, double *sumsq, void *stream) {
    int grid = (int)std::min<size_t>(4096, (n + 255) / 256);
    if (grid < 1) grid = 1;
    residual_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(seis, obs, res, n, sumsq);
    return (int)cudaGetLastError();
}

}  // namespace s2d

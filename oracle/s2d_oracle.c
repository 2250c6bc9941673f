/*
 * s2d_oracle.c -- CPU restatement of SeisAcoMod2D's per-shot forward path.
 *
 * TEST INFRASTRUCTURE (the checker, never the product): loaded only by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.
 *
 * Every routine names the reference lines it restates.  Paths are relative to
 * the SeisAcoMod2D source tree:
 *   CM  = src/src_cpu/cpumodelling.cpp
 *   CK  = src/src_cpu/cpu_modelling_kernels.cpp
 * Arithmetic in the ORC_F64 variant keeps the reference's float/double mix and
 * operation order, so its seismograms are expected to equal the reference's
 * bit for bit; the ORC_F32 variant runs the same steps in FP32.
 */
#include "s2d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.141592654 /* CM:9, CK:7 */

/* Threads of the gradient's loops (orc_set_threads).  ORC_PAR_FOR splits a
 * loop over cells whose updates are independent, or over row blocks of a
 * scatter whose additions into each cell keep their serial order: the same
 * bits for every thread count.  One thread runs the loops serially. */
static int g_threads = 1;
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
#define ORC_PAR_FOR _Pragma("omp parallel for if (g_threads > 1) num_threads(g_threads) schedule(static)")
#define ORC_ROWS 64 /* rows per block of the x-direction scatters */

/* 4th-order staggered coefficients, CK:9-10.  The reference's macro
 * "-1.0f/24.0f" is a float quotient, so a1 carries float rounding. */
static const float ORC_A0 = 1.125f;
static const float ORC_A1 = -1.0f / 24.0f;

void orc_derive(const orc_params *p, orc_derived *d) {
    /* CM:168-193 */
    float inv_dx = 1.0f / p->dx, inv_dz = 1.0f / p->dz;
    d->fd_nt = (int)ceilf(p->rec_len / p->fd_dt);
    d->real_nt = (int)ceilf(p->rec_len / p->real_dt);
    d->dtdx = (double)(p->fd_dt * inv_dx);
    d->dtdz = (double)(p->fd_dt * inv_dz);
    d->dt_factor = (int)(p->real_dt / p->fd_dt);
    /* CM:183: sqrt(6.0f) resolves to the float overload of std::sqrt. */
    double td = sqrtf(6.0f) / (ORC_PI * p->fm);
    d->nts = (int)(5.0f * td / p->fd_dt) + 1;
    if (d->nts > d->fd_nt) d->nts = d->fd_nt;
    d->nnz = 2 * p->nb + p->nz;
    d->nnx = 2 * p->nb + p->nx;
}

void orc_ricker(const orc_params *p, const orc_derived *d, double *w) {
    /* CK:33-62 with iss == 2 */
    double t0 = 1.5 * sqrt(6.0) / (ORC_PI * (double)p->fm);
    for (int i = 0; i < d->nts; i++) {
        double t = (double)(i * p->fd_dt);
        double a = ORC_PI * (double)p->fm * (t - t0);
        double a2 = a * a;
        w[i] = (1.0f - 2.0f * a2) * exp(-a2);
    }
}

int orc_cell(const orc_params *p, float x, float z) {
    /* CM:288-289 and CK:15-22 */
    int nnz = 2 * p->nb + p->nz;
    float inv_dx = 1.0f / p->dx, inv_dz = 1.0f / p->dz;
    int ix = (int)(x * inv_dx), iz = (int)(z * inv_dz);
    return nnz * (ix + p->nb) + (iz + p->nb);
}

/* CM:39-60: copy [nx1][nz1] into the padded grid and replicate the edges. */
static void expand(float *b, const float *a, int nb, int nnz, int nnx, int nz1, int nx1) {
    for (int ix = 0; ix < nx1; ix++)
        for (int iz = 0; iz < nz1; iz++) b[(nb + ix) * nnz + (nb + iz)] = a[ix * nz1 + iz];
    for (int ix = 0; ix < nnx; ix++) {
        for (int iz = 0; iz < nb; iz++) b[ix * nnz + iz] = b[ix * nnz + nb];
        for (int iz = nz1 + nb; iz < nnz; iz++) b[ix * nnz + iz] = b[ix * nnz + nb + nz1 - 1];
    }
    for (int iz = 0; iz < nnz; iz++) {
        for (int ix = 0; ix < nb; ix++) b[ix * nnz + iz] = b[nb * nnz + iz];
        for (int ix = nb + nx1; ix < nnx; ix++) b[ix * nnz + iz] = b[(nb + nx1 - 1) * nnz + iz];
    }
}

/* CK:64-121: kappa = vp^2 rho (double), buoyancy b = 1/rho, and its two
 * staggered averages.  bz (reference bu1) averages along z; its last row is
 * read from bx before bx is filled, so it is 0 (CK:100).  bx (reference bu2)
 * averages along x; its last column copies bz of column nnx-2 (CK:115-119). */
static void stagger(const float *vpe, const float *rhoe, float *bue, float *bx, float *bz,
                    double *kappa, int nnz, int nnx) {
    size_t N = (size_t)nnz * nnx;
    memset(bx, 0, N * sizeof(float));
    memset(bz, 0, N * sizeof(float));
    for (size_t id = 0; id < N; id++) {
        double vp2 = (double)vpe[id] * (double)vpe[id];
        kappa[id] = vp2 * (double)rhoe[id];
        bue[id] = rhoe[id] > 0.0f ? 1.0f / rhoe[id] : 10000000000.0f;
    }
    for (int i2 = 0; i2 < nnx; i2++) {
        for (int i1 = 0; i1 < nnz - 1; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            bz[id] = 0.5f * (bue[id + 1] + bue[id]);
        }
        bz[(size_t)i2 * nnz + nnz - 1] = bx[(size_t)i2 * nnz + nnz - 2];
    }
    for (int i2 = 0; i2 < nnx - 1; i2++)
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            bx[id] = 0.5f * (bue[id + nnz] + bue[id]);
        }
    for (int i1 = 0; i1 < nnz; i1++) bx[(size_t)(nnx - 1) * nnz + i1] = bz[(size_t)(nnx - 2) * nnz + i1];
}

/* Pressure-release (free) surface at the first model row, the vacuum form:
 * kappa = 0 on padded rows 0..nb keeps px = pz = p = 0 there, so the
 * surface row carries p = 0 and the rows above it are vacuum.  A source on
 * those rows injects nothing (its amplitude scales with kappa at the source).
 * No counterpart in the reference, which parses "Free surface" and ignores it
 * (json_parser.cpp:236-244; Instructions: "Free surface yet not implemented"). */
static void free_surface_rows(double *kappa, int nb, int nnz, int nnx) {
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz <= nb && iz < nnz; iz++) kappa[(size_t)iz + (size_t)ix * nnz] = 0.0;
}

/* CK:123-153: sponge at integer nodes.  spg uses the float overload of exp
 * (its argument is float), spg1 the double one. */
static void sponge_a(float fac, float *damp, float *damp1, int nb, int n) {
    float *spg = (float *)calloc(nb + 1, sizeof(float));
    float *spg1 = (float *)calloc(nb + 1, sizeof(float));
    for (int i = 0; i < nb; i++) {
        float x = (float)(nb - (i + 1));
        float t = fac * x;
        spg[i] = expf(-(t * t));
        spg1[i] = (float)exp(-0.5 * (t * t));
    }
    for (int i = 0; i < nb; i++) {
        damp[i] = spg[i];
        damp1[i] = spg1[i];
        damp[nb + n + i] = spg[nb - i - 1];
        damp1[nb + n + i] = spg1[nb - i - 1];
    }
    for (int i = 0; i < n; i++) {
        damp[i + nb] = 1.0f;
        damp1[i + nb] = 1.0f;
    }
    free(spg);
    free(spg1);
}

/* CK:155-199: sponge at half nodes. */
static void sponge_b(float fac, float *damp, float *damp1, int nb, int n) {
    float *spg = (float *)calloc(nb + 1, sizeof(float));
    float *spg1 = (float *)calloc(nb + 1, sizeof(float));
    for (int i = 0; i < nb - 1; i++) {
        float x = (float)(nb - 1 - (i + 1)) + 0.5f;
        float t = fac * x;
        spg[i] = expf(-(t * t));
        spg1[i] = (float)exp(-0.5 * (t * t));
    }
    for (int i = 0; i < nb - 1; i++) {
        damp[i] = spg[i];
        damp1[i] = spg1[i];
    }
    for (int i = 0; i < n + 1; i++) {
        damp[i + nb - 1] = 1.0f;
        damp1[i + nb - 1] = 1.0f;
    }
    for (int i = 0; i < nb; i++) {
        float x = (float)((i + 1) - 1) + 0.5f;
        float t = fac * x;
        spg[i] = expf(-(t * t));
        spg1[i] = (float)exp(-0.5 * (t * t));
    }
    for (int i = 0; i < nb; i++) {
        damp[nb + n + i] = spg[i];
        damp1[nb + n + i] = spg1[i];
    }
    free(spg);
    free(spg1);
}

/* ---------------- FP64 step: CM:115-156 with CK:201-368 ------------------ */

typedef struct {
    int nnx, nnz;
    size_t N;
    double *p, *px, *pz, *vx, *vz, *d1, *d2;
    const double *kw1, *kw2, *bw1, *bw2; /* CM:270-281 */
    const float *damp1a, *damp2a, *damp1b, *damp2b;
} f64_state;

static void f64_step(f64_state *s, int isrc, double src_add, int inject) {
    const int nnz = s->nnz, nnx = s->nnx;
    const size_t N = s->N;
    double *d1 = s->d1, *d2 = s->d2;
    memset(d1, 0, N * sizeof(double));
    memset(d2, 0, N * sizeof(double));
    /* CK:201-229  der2 = D-x vx */
    for (int i2 = 2; i2 < nnx - 1; i2++)
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            d2[id] = ORC_A0 * (s->vx[id] - s->vx[id - nnz]) + ORC_A1 * (s->vx[id + nnz] - s->vx[id - 2 * nnz]);
        }
    for (int i1 = 0; i1 < nnz; i1++) {
        size_t id = (size_t)i1 + (size_t)1 * nnz;
        d2[id] = s->vx[id] - s->vx[id - nnz];
        id = (size_t)i1 + (size_t)(nnx - 1) * nnz;
        d2[id] = s->vx[id] - s->vx[id - nnz];
    }
    /* CK:231-258  der1 = D-z vz */
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 2; i1 < nnz - 1; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            d1[id] = ORC_A0 * (s->vz[id] - s->vz[id - 1]) + ORC_A1 * (s->vz[id + 1] - s->vz[id - 2]);
        }
    for (int i2 = 0; i2 < nnx; i2++) {
        size_t id = (size_t)(nnz - 1) + (size_t)i2 * nnz;
        d1[id] = s->vz[id] - s->vz[id - 1];
        id = (size_t)1 + (size_t)i2 * nnz;
        d1[id] = s->vz[id] - s->vz[id - 1];
    }
    /* CK:335-351  split-field pressure with sponge */
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            s->px[id] = s->damp2a[i2] * s->px[id] + s->kw2[id] * d2[id];
            s->pz[id] = s->damp1a[i1] * s->pz[id] + s->kw1[id] * d1[id];
        }
    /* CM:136-140  source */
    if (inject) s->px[isrc] = s->px[isrc] + src_add;
    /* CK:318-333 */
    for (size_t id = 0; id < N; id++) s->p[id] = s->px[id] + s->pz[id];
    memset(d1, 0, N * sizeof(double));
    memset(d2, 0, N * sizeof(double));
    /* CK:260-287  der2 = D+x p */
    for (int i2 = 1; i2 < nnx - 2; i2++)
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            d2[id] = ORC_A0 * (s->p[id + nnz] - s->p[id]) + ORC_A1 * (s->p[id + 2 * nnz] - s->p[id - nnz]);
        }
    for (int i1 = 0; i1 < nnz; i1++) {
        size_t id = (size_t)i1;
        d2[id] = s->p[id + nnz] - s->p[id];
        id = (size_t)i1 + (size_t)(nnx - 2) * nnz;
        d2[id] = s->p[id + nnz] - s->p[id];
    }
    /* CK:289-316  der1 = D+z p */
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 1; i1 < nnz - 2; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            d1[id] = ORC_A0 * (s->p[id + 1] - s->p[id]) + ORC_A1 * (s->p[id + 2] - s->p[id - 1]);
        }
    for (int i2 = 0; i2 < nnx; i2++) {
        size_t id = (size_t)(nnz - 2) + (size_t)i2 * nnz;
        d1[id] = s->p[id + 1] - s->p[id];
        id = (size_t)i2 * nnz;
        d1[id] = s->p[id + 1] - s->p[id];
    }
    /* CK:353-368 */
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            s->vx[id] = s->damp2b[i2] * s->vx[id] + s->bw2[id] * d2[id];
            s->vz[id] = s->damp1b[i1] * s->vz[id] + s->bw1[id] * d1[id];
        }
}

/* ---------------- FP32 step: same scheme, FP32 arithmetic ---------------- */

/* The same four derivative operators, with the per-row coefficient pair
 * (c0, c1) that encodes the reference's edge rows: 4th order inside, plain
 * difference on the rows CK:217-227 / 247-256 / 276-285 / 305-314 list, and
 * zero on the row each operator leaves at 0. */
static inline void dm_coef(int i, int n, float *c0, float *c1) { /* D- : rows [2,n-2] 4th, 1 and n-1 2nd, 0 zero */
    if (i >= 2 && i <= n - 2) { *c0 = ORC_A0; *c1 = ORC_A1; }
    else if (i == 1 || i == n - 1) { *c0 = 1.0f; *c1 = 0.0f; }
    else { *c0 = 0.0f; *c1 = 0.0f; }
}
static inline void dp_coef(int i, int n, float *c0, float *c1) { /* D+ : rows [1,n-3] 4th, 0 and n-2 2nd, n-1 zero */
    if (i >= 1 && i <= n - 3) { *c0 = ORC_A0; *c1 = ORC_A1; }
    else if (i == 0 || i == n - 2) { *c0 = 1.0f; *c1 = 0.0f; }
    else { *c0 = 0.0f; *c1 = 0.0f; }
}

typedef struct {
    int nnx, nnz;
    size_t N;
    float *p, *px, *pz, *vx, *vz;
    const float *kappa, *bx, *bz;
    const float *damp1a, *damp2a, *damp1b, *damp2b;
    const float *kxa, *kza, *kxb, *kzb; /* dt/d * damp?1 folded per column / row */
} f32_state;

#define AT(a, ix, iz) ((ix) < 0 || (ix) >= nnx || (iz) < 0 || (iz) >= nnz ? 0.0f : (a)[(size_t)(ix) * nnz + (iz)])

static void f32_step(f32_state *s, int isrc, float src_add, int inject) {
    const int nnz = s->nnz, nnx = s->nnx;
    for (int ix = 0; ix < nnx; ix++) {
        float cx0, cx1;
        dm_coef(ix, nnx, &cx0, &cx1);
        for (int iz = 0; iz < nnz; iz++) {
            float cz0, cz1;
            dm_coef(iz, nnz, &cz0, &cz1);
            size_t id = (size_t)ix * nnz + iz;
            float dvx = cx0 * (AT(s->vx, ix, iz) - AT(s->vx, ix - 1, iz)) + cx1 * (AT(s->vx, ix + 1, iz) - AT(s->vx, ix - 2, iz));
            float dvz = cz0 * (AT(s->vz, ix, iz) - AT(s->vz, ix, iz - 1)) + cz1 * (AT(s->vz, ix, iz + 1) - AT(s->vz, ix, iz - 2));
            float k = s->kappa[id];
            if (s->damp2a[ix] == 1.0f && s->damp1a[iz] == 1.0f) {
                /* Both split fields undamped: they only enter through
                 * p = px + pz, so the cell carries p alone (px = p, pz = 0),
                 * as the CUDA kernels do.  Same scheme in exact arithmetic. */
                float t = s->kxa[ix] * dvx + s->kza[iz] * dvz;
                s->px[id] = s->px[id] + k * t;
                s->pz[id] = 0.0f;
            } else {
                s->px[id] = s->damp2a[ix] * s->px[id] + (s->kxa[ix] * k) * dvx;
                s->pz[id] = s->damp1a[iz] * s->pz[id] + (s->kza[iz] * k) * dvz;
            }
        }
    }
    if (inject) s->px[isrc] = s->px[isrc] + src_add;
    for (size_t id = 0; id < s->N; id++) s->p[id] = s->px[id] + s->pz[id];
    for (int ix = 0; ix < nnx; ix++) {
        float cx0, cx1;
        dp_coef(ix, nnx, &cx0, &cx1);
        for (int iz = 0; iz < nnz; iz++) {
            float cz0, cz1;
            dp_coef(iz, nnz, &cz0, &cz1);
            size_t id = (size_t)ix * nnz + iz;
            float dpx = cx0 * (AT(s->p, ix + 1, iz) - AT(s->p, ix, iz)) + cx1 * (AT(s->p, ix + 2, iz) - AT(s->p, ix - 1, iz));
            float dpz = cz0 * (AT(s->p, ix, iz + 1) - AT(s->p, ix, iz)) + cz1 * (AT(s->p, ix, iz + 2) - AT(s->p, ix, iz - 1));
            s->vx[id] = s->damp2b[ix] * s->vx[id] + (s->kxb[ix] * s->bx[id]) * dpx;
            s->vz[id] = s->damp1b[iz] * s->vz[id] + (s->kzb[iz] * s->bz[id]) * dpz;
        }
    }
}
#undef AT

/* ------------- 8th-order operator (no counterpart in the reference) -------
 *
 * "Order of FD Operator" = 8.  The reference parses the key and runs its step
 * only for 4 (cpumodelling.cpp:121, `if (NJ == 4)`), so this is new
 * capability with no reference output.  Staggered-grid 8th-order Taylor
 * coefficients (c1..c4 = 1225/1024, -245/3072, 49/5120, -5/7168, rounded to
 * float), in the forms
 *   D- f[i] = sum_k c_k (f[i+k-1] - f[i-k])     (taps i-4 .. i+3)
 *   D+ f[i] = sum_k c_k (f[i+k] - f[i-k+1])     (taps i-3 .. i+4)
 * Rows whose taps would leave the grid fall back to the reference's operator:
 * its 4th-order pair (a0, a1), its plain difference, its zero row. */
static const float ORC_C81 = 1225.0f / 1024.0f;
static const float ORC_C82 = -245.0f / 3072.0f;
static const float ORC_C83 = 49.0f / 5120.0f;
static const float ORC_C84 = -5.0f / 7168.0f;

static inline void dm8_coef(int i, int n, float c[4]) { /* D-: 8th on [4, n-4], then the reference's rows */
    if (i >= 4 && i <= n - 4) { c[0] = ORC_C81; c[1] = ORC_C82; c[2] = ORC_C83; c[3] = ORC_C84; return; }
    c[2] = c[3] = 0.0f;
    dm_coef(i, n, &c[0], &c[1]);
}
static inline void dp8_coef(int i, int n, float c[4]) { /* D+: 8th on [3, n-5], then the reference's rows */
    if (i >= 3 && i <= n - 5) { c[0] = ORC_C81; c[1] = ORC_C82; c[2] = ORC_C83; c[3] = ORC_C84; return; }
    c[2] = c[3] = 0.0f;
    dp_coef(i, n, &c[0], &c[1]);
}

/* FP64 step, split fields everywhere as the reference's FP64 path (CM:115-156
 * with the 8th-order operators). */
static void f64_step8(f64_state *s, int isrc, double src_add, int inject) {
    const int nnz = s->nnz, nnx = s->nnx;
#define AT64(a, ix, iz) ((ix) < 0 || (ix) >= nnx || (iz) < 0 || (iz) >= nnz ? 0.0 : (a)[(size_t)(ix) * nnz + (iz)])
    for (int ix = 0; ix < nnx; ix++) {
        float cx[4];
        dm8_coef(ix, nnx, cx);
        for (int iz = 0; iz < nnz; iz++) {
            float cz[4];
            dm8_coef(iz, nnz, cz);
            double dvx = 0.0, dvz = 0.0;
            for (int k = 0; k < 4; k++) {
                dvx += (double)cx[k] * (AT64(s->vx, ix + k, iz) - AT64(s->vx, ix - 1 - k, iz));
                dvz += (double)cz[k] * (AT64(s->vz, ix, iz + k) - AT64(s->vz, ix, iz - 1 - k));
            }
            size_t id = (size_t)ix * nnz + iz;
            s->px[id] = s->damp2a[ix] * s->px[id] + s->kw2[id] * dvx;
            s->pz[id] = s->damp1a[iz] * s->pz[id] + s->kw1[id] * dvz;
        }
    }
    if (inject) s->px[isrc] = s->px[isrc] + src_add;
    for (size_t id = 0; id < s->N; id++) s->p[id] = s->px[id] + s->pz[id];
    for (int ix = 0; ix < nnx; ix++) {
        float cx[4];
        dp8_coef(ix, nnx, cx);
        for (int iz = 0; iz < nnz; iz++) {
            float cz[4];
            dp8_coef(iz, nnz, cz);
            double dpx = 0.0, dpz = 0.0;
            for (int k = 0; k < 4; k++) {
                dpx += (double)cx[k] * (AT64(s->p, ix + 1 + k, iz) - AT64(s->p, ix - k, iz));
                dpz += (double)cz[k] * (AT64(s->p, ix, iz + 1 + k) - AT64(s->p, ix, iz - k));
            }
            size_t id = (size_t)ix * nnz + iz;
            s->vx[id] = s->damp2b[ix] * s->vx[id] + s->bw2[id] * dpx;
            s->vz[id] = s->damp1b[iz] * s->vz[id] + s->bw1[id] * dpz;
        }
    }
#undef AT64
}

/* FP32 step with the CUDA kernel's rounding: every derivative
 * fma(c1, d1, fma(c2, d2, fma(c3, d3, c4*d4))), every update
 * fma(damping, field, (coefficient * material) * derivative), merged cells
 * (both pressure dampings 1) carrying p alone as in f32_step. */
#define AT(a, ix, iz) ((ix) < 0 || (ix) >= nnx || (iz) < 0 || (iz) >= nnz ? 0.0f : (a)[(size_t)(ix) * nnz + (iz)])
static inline float dif8(const float c[4], float d1, float d2, float d3, float d4) {
    return fmaf(c[0], d1, fmaf(c[1], d2, fmaf(c[2], d3, c[3] * d4)));
}
static void f32_step8(f32_state *s, int isrc, float src_add, int inject) {
    const int nnz = s->nnz, nnx = s->nnx;
    for (int ix = 0; ix < nnx; ix++) {
        float cx[4];
        dm8_coef(ix, nnx, cx);
        for (int iz = 0; iz < nnz; iz++) {
            float cz[4];
            dm8_coef(iz, nnz, cz);
            size_t id = (size_t)ix * nnz + iz;
            const float *vx = s->vx, *vz = s->vz;
            float dvx = dif8(cx, AT(vx, ix, iz) - AT(vx, ix - 1, iz), AT(vx, ix + 1, iz) - AT(vx, ix - 2, iz),
                             AT(vx, ix + 2, iz) - AT(vx, ix - 3, iz), AT(vx, ix + 3, iz) - AT(vx, ix - 4, iz));
            float dvz = dif8(cz, AT(vz, ix, iz) - AT(vz, ix, iz - 1), AT(vz, ix, iz + 1) - AT(vz, ix, iz - 2),
                             AT(vz, ix, iz + 2) - AT(vz, ix, iz - 3), AT(vz, ix, iz + 3) - AT(vz, ix, iz - 4));
            float k = s->kappa[id];
            if (s->damp2a[ix] == 1.0f && s->damp1a[iz] == 1.0f) {
                float t = fmaf(s->kxa[ix], dvx, s->kza[iz] * dvz);
                s->px[id] = fmaf(k, t, s->px[id]);
                s->pz[id] = 0.0f;
            } else {
                s->px[id] = fmaf(s->damp2a[ix], s->px[id], (s->kxa[ix] * k) * dvx);
                s->pz[id] = fmaf(s->damp1a[iz], s->pz[id], (s->kza[iz] * k) * dvz);
            }
        }
    }
    if (inject) s->px[isrc] = s->px[isrc] + src_add;
    for (size_t id = 0; id < s->N; id++) s->p[id] = s->px[id] + s->pz[id];
    for (int ix = 0; ix < nnx; ix++) {
        float cx[4];
        dp8_coef(ix, nnx, cx);
        for (int iz = 0; iz < nnz; iz++) {
            float cz[4];
            dp8_coef(iz, nnz, cz);
            size_t id = (size_t)ix * nnz + iz;
            const float *p = s->p;
            float dpx = dif8(cx, AT(p, ix + 1, iz) - AT(p, ix, iz), AT(p, ix + 2, iz) - AT(p, ix - 1, iz),
                             AT(p, ix + 3, iz) - AT(p, ix - 2, iz), AT(p, ix + 4, iz) - AT(p, ix - 3, iz));
            float dpz = dif8(cz, AT(p, ix, iz + 1) - AT(p, ix, iz), AT(p, ix, iz + 2) - AT(p, ix, iz - 1),
                             AT(p, ix, iz + 3) - AT(p, ix, iz - 2), AT(p, ix, iz + 4) - AT(p, ix, iz - 3));
            s->vx[id] = fmaf(s->damp2b[ix], s->vx[id], (s->kxb[ix] * s->bx[id]) * dpx);
            s->vz[id] = fmaf(s->damp1b[iz], s->vz[id], (s->kzb[iz] * s->bz[id]) * dpz);
        }
    }
}
#undef AT

/* ------------------------------ driver ---------------------------------- */

int orc_forward(const orc_params *prm, int precision,
                const float *vp, const float *rho,
                float sx, float sz, int nrec, const float *gx, const float *gz,
                const double *wavelet, int nwav, int kt_stop,
                float *seis, double *state_out) {
    if (!prm || !vp || !rho || nrec < 0 || (nrec > 0 && (!gx || !gz || !seis))) return -1;
    if (prm->nx < 1 || prm->nz < 1 || prm->nb < 2) return -1;
    if (precision != ORC_F64 && precision != ORC_F32) return -1;
    if (prm->fd_order != 0 && prm->fd_order != 4 && prm->fd_order != 8) return -1;
    const int o8 = prm->fd_order == 8;
    orc_derived d;
    orc_derive(prm, &d);
    if (d.dt_factor < 1 || d.fd_nt < 1) return -2;
    const int nnx = d.nnx, nnz = d.nnz, nb = prm->nb;
    const size_t N = (size_t)nnx * nnz;

    /* CM:207-230 */
    float *vel = (float *)calloc(N, sizeof(float));
    float *den = (float *)calloc(N, sizeof(float));
    float *bue = (float *)calloc(N, sizeof(float));
    float *bx = (float *)calloc(N, sizeof(float));
    float *bz = (float *)calloc(N, sizeof(float));
    double *kappa = (double *)calloc(N, sizeof(double));
    expand(vel, vp, nb, nnz, nnx, prm->nz, prm->nx);
    expand(den, rho, nb, nnz, nnx, prm->nz, prm->nx);
    stagger(vel, den, bue, bx, bz, kappa, nnz, nnx);
    if (prm->free_surface) free_surface_rows(kappa, nb, nnz, nnx);

    /* CM:233-234 (plus the one-past-the-end sample read at kt == nts, CM:136,
     * taken as 0 here) */
    int nw = wavelet ? nwav : d.nts;
    double *w = (double *)calloc((size_t)(nw > 0 ? nw : 0) + 1, sizeof(double));
    if (wavelet) memcpy(w, wavelet, (size_t)nw * sizeof(double));
    else orc_ricker(prm, &d, w);

    /* CM:254-259 */
    float *damp2a = (float *)calloc(nnx, sizeof(float)), *damp2a1 = (float *)calloc(nnx, sizeof(float));
    float *damp2b = (float *)calloc(nnx, sizeof(float)), *damp2b1 = (float *)calloc(nnx, sizeof(float));
    float *damp1a = (float *)calloc(nnz, sizeof(float)), *damp1a1 = (float *)calloc(nnz, sizeof(float));
    float *damp1b = (float *)calloc(nnz, sizeof(float)), *damp1b1 = (float *)calloc(nnz, sizeof(float));
    const float fac = 0.05f;
    sponge_a(fac, damp2a, damp2a1, nb, prm->nx);
    sponge_b(fac, damp2b, damp2b1, nb, prm->nx);
    sponge_a(fac, damp1a, damp1a1, nb, prm->nz);
    sponge_b(fac, damp1b, damp1b1, nb, prm->nz);

    /* CM:284-292, 329-338 */
    int isrc = orc_cell(prm, sx, sz);
    int *gcell = (int *)calloc((size_t)nrec + 1, sizeof(int));
    for (int g = 0; g < nrec; g++) gcell[g] = orc_cell(prm, gx[g], gz[g]);
    if (isrc < 0 || (size_t)isrc >= N) goto bad_pos;
    for (int g = 0; g < nrec; g++)
        if (gcell[g] < 0 || (size_t)gcell[g] >= N) goto bad_pos;

    int nsteps = (kt_stop > 0 && kt_stop < d.fd_nt) ? kt_stop : d.fd_nt;
    float *temp = (float *)calloc((size_t)nrec * d.real_nt + 1, sizeof(float));
    const float dxdz = prm->dx * prm->dz;

    if (precision == ORC_F64) {
        double *kw1 = (double *)malloc(N * sizeof(double)), *kw2 = (double *)malloc(N * sizeof(double));
        double *bw1 = (double *)malloc(N * sizeof(double)), *bw2 = (double *)malloc(N * sizeof(double));
        /* CM:270-281 */
        for (int ix = 0; ix < nnx; ix++)
            for (int iz = 0; iz < nnz; iz++) {
                size_t id = (size_t)iz + (size_t)ix * nnz;
                kw2[id] = d.dtdx * kappa[id] * damp2a1[ix];
                kw1[id] = d.dtdz * kappa[id] * damp1a1[iz];
                bw2[id] = d.dtdx * bx[id] * damp2b1[ix];
                bw1[id] = d.dtdz * bz[id] * damp1b1[iz];
            }
        f64_state s = {nnx, nnz, N, NULL, NULL, NULL, NULL, NULL, NULL, NULL,
                       kw1, kw2, bw1, bw2, damp1a, damp2a, damp1b, damp2b};
        double **f[7] = {&s.p, &s.px, &s.pz, &s.vx, &s.vz, &s.d1, &s.d2};
        for (int k = 0; k < 7; k++) *f[k] = (double *)calloc(N, sizeof(double));
        for (int kt = 0; kt < nsteps; kt++) {
            /* CM:136-140 */
            double wk = kt < nw ? w[kt] : 0.0;
            double add = prm->fd_dt * wk * kappa[isrc] / (dxdz);
            if (o8) f64_step8(&s, isrc, add, kt <= d.nts);
            else f64_step(&s, isrc, add, kt <= d.nts);
            /* CM:356-360 */
            if ((kt + 1) % d.dt_factor == 0) {
                int it = (kt + 1) / d.dt_factor - 1;
                if (it < d.real_nt)
                    for (int g = 0; g < nrec; g++) temp[(size_t)it * nrec + g] = (float)s.p[gcell[g]];
            }
        }
        if (state_out) {
            memcpy(state_out + 0 * N, s.px, N * sizeof(double));
            memcpy(state_out + 1 * N, s.pz, N * sizeof(double));
            memcpy(state_out + 2 * N, s.vx, N * sizeof(double));
            memcpy(state_out + 3 * N, s.vz, N * sizeof(double));
            memcpy(state_out + 4 * N, s.p, N * sizeof(double));
        }
        for (int k = 0; k < 7; k++) free(*f[k]);
        free(kw1); free(kw2); free(bw1); free(bw2);
    } else {
        float *kf = (float *)malloc(N * sizeof(float));
        for (size_t id = 0; id < N; id++) kf[id] = (float)kappa[id];
        float *kxa = (float *)malloc(nnx * sizeof(float)), *kxb = (float *)malloc(nnx * sizeof(float));
        float *kza = (float *)malloc(nnz * sizeof(float)), *kzb = (float *)malloc(nnz * sizeof(float));
        for (int ix = 0; ix < nnx; ix++) { kxa[ix] = (float)(d.dtdx * damp2a1[ix]); kxb[ix] = (float)(d.dtdx * damp2b1[ix]); }
        for (int iz = 0; iz < nnz; iz++) { kza[iz] = (float)(d.dtdz * damp1a1[iz]); kzb[iz] = (float)(d.dtdz * damp1b1[iz]); }
        f32_state s = {nnx, nnz, N, NULL, NULL, NULL, NULL, NULL, kf, bx, bz,
                       damp1a, damp2a, damp1b, damp2b, kxa, kza, kxb, kzb};
        float **f[5] = {&s.p, &s.px, &s.pz, &s.vx, &s.vz};
        for (int k = 0; k < 5; k++) *f[k] = (float *)calloc(N, sizeof(float));
        for (int kt = 0; kt < nsteps; kt++) {
            double wk = kt < nw ? w[kt] : 0.0;
            float add = (float)(prm->fd_dt * wk * kappa[isrc] / (dxdz));
            if (o8) f32_step8(&s, isrc, add, kt <= d.nts);
            else f32_step(&s, isrc, add, kt <= d.nts);
            if ((kt + 1) % d.dt_factor == 0) {
                int it = (kt + 1) / d.dt_factor - 1;
                if (it < d.real_nt)
                    for (int g = 0; g < nrec; g++) temp[(size_t)it * nrec + g] = s.p[gcell[g]];
            }
        }
        if (state_out) {
            float *src[5] = {s.px, s.pz, s.vx, s.vz, s.p};
            for (int k = 0; k < 5; k++)
                for (size_t id = 0; id < N; id++) state_out[k * N + id] = src[k][id];
        }
        for (int k = 0; k < 5; k++) free(*f[k]);
        free(kf); free(kxa); free(kxb); free(kza); free(kzb);
    }

    /* CK:370-381: [real_nt][nrec] -> [nrec][real_nt] */
    for (int t = 0; t < d.real_nt; t++)
        for (int g = 0; g < nrec; g++) seis[(size_t)g * d.real_nt + t] = temp[(size_t)t * nrec + g];
    free(temp);
    free(vel); free(den); free(bue); free(bx); free(bz); free(kappa); free(w); free(gcell);
    free(damp2a); free(damp2a1); free(damp2b); free(damp2b1);
    free(damp1a); free(damp1a1); free(damp1b); free(damp1b1);
    return 0;

bad_pos:
    free(vel); free(den); free(bue); free(bx); free(bz); free(kappa); free(w); free(gcell);
    free(damp2a); free(damp2a1); free(damp2b); free(damp2b1);
    free(damp1a); free(damp1a1); free(damp1b); free(damp1b1);
    return -3;
}

/* ------------------------- FP64 discrete adjoint -------------------------
 *
 * The forward step of f64_step, written with its intermediate derivatives
 *   a = Gx vx, c = Gz vz                  (CK:201-258, old velocities)
 *   px' = damp2a px + kw2 a (+ source), pz' = damp1a pz + kw1 c
 *   p' = px' + pz',  g = Hx p', h = Hz p'  (CK:260-316)
 *   vx' = damp2b vx + bw2 g,  vz' = damp1b vz + bw1 h
 * is linear in the state, so its adjoint runs the same stages backwards with
 * every operator transposed.  The transposes below scatter each row of the
 * forward operator exactly as the forward code defines that row, so they are
 * the transposes of the reference's operators including its edge rows. */

/* out += Gx^T mu, Gx = D-x of CK:201-229 */
static void gxT_add(const double *mu, double *out, int nnz, int nnx) {
    const int nblk = (nnz + ORC_ROWS - 1) / ORC_ROWS;
    ORC_PAR_FOR
    for (int b = 0; b < nblk; b++)
        for (int i2 = 2; i2 < nnx - 1; i2++)
            for (int i1 = b * ORC_ROWS; i1 < nnz && i1 < (b + 1) * ORC_ROWS; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                double m = mu[id];
                out[id] += ORC_A0 * m;
                out[id - nnz] -= ORC_A0 * m;
                out[id + nnz] += ORC_A1 * m;
                out[id - 2 * nnz] -= ORC_A1 * m;
            }
    for (int i1 = 0; i1 < nnz; i1++) {
        size_t id = (size_t)i1 + (size_t)1 * nnz;
        out[id] += mu[id];
        out[id - nnz] -= mu[id];
        id = (size_t)i1 + (size_t)(nnx - 1) * nnz;
        out[id] += mu[id];
        out[id - nnz] -= mu[id];
    }
}
/* out += Gz^T mu, Gz = D-z of CK:231-258 */
static void gzT_add(const double *mu, double *out, int nnz, int nnx) {
    ORC_PAR_FOR
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 2; i1 < nnz - 1; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            double m = mu[id];
            out[id] += ORC_A0 * m;
            out[id - 1] -= ORC_A0 * m;
            out[id + 1] += ORC_A1 * m;
            out[id - 2] -= ORC_A1 * m;
        }
    for (int i2 = 0; i2 < nnx; i2++) {
        size_t id = (size_t)(nnz - 1) + (size_t)i2 * nnz;
        out[id] += mu[id];
        out[id - 1] -= mu[id];
        id = (size_t)1 + (size_t)i2 * nnz;
        out[id] += mu[id];
        out[id - 1] -= mu[id];
    }
}
/* out += Hx^T mu, Hx = D+x of CK:260-287 */
static void hxT_add(const double *mu, double *out, int nnz, int nnx) {
    const int nblk = (nnz + ORC_ROWS - 1) / ORC_ROWS;
    ORC_PAR_FOR
    for (int b = 0; b < nblk; b++)
        for (int i2 = 1; i2 < nnx - 2; i2++)
            for (int i1 = b * ORC_ROWS; i1 < nnz && i1 < (b + 1) * ORC_ROWS; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                double m = mu[id];
                out[id + nnz] += ORC_A0 * m;
                out[id] -= ORC_A0 * m;
                out[id + 2 * nnz] += ORC_A1 * m;
                out[id - nnz] -= ORC_A1 * m;
            }
    for (int i1 = 0; i1 < nnz; i1++) {
        size_t id = (size_t)i1;
        out[id + nnz] += mu[id];
        out[id] -= mu[id];
        id = (size_t)i1 + (size_t)(nnx - 2) * nnz;
        out[id + nnz] += mu[id];
        out[id] -= mu[id];
    }
}
/* out += Hz^T mu, Hz = D+z of CK:289-316 */
static void hzT_add(const double *mu, double *out, int nnz, int nnx) {
    ORC_PAR_FOR
    for (int i2 = 0; i2 < nnx; i2++)
        for (int i1 = 1; i1 < nnz - 2; i1++) {
            size_t id = (size_t)i1 + (size_t)i2 * nnz;
            double m = mu[id];
            out[id + 1] += ORC_A0 * m;
            out[id] -= ORC_A0 * m;
            out[id + 2] += ORC_A1 * m;
            out[id - 1] -= ORC_A1 * m;
        }
    for (int i2 = 0; i2 < nnx; i2++) {
        size_t id = (size_t)(nnz - 2) + (size_t)i2 * nnz;
        out[id + 1] += mu[id];
        out[id] -= mu[id];
        id = (size_t)i2 * nnz;
        out[id + 1] += mu[id];
        out[id] -= mu[id];
    }
}

/* d = G f for the four forward operators (same code as f64_step). */
static void op_apply(int which, const double *f, double *d, int nnz, int nnx) {
    size_t N = (size_t)nnz * nnx;
    memset(d, 0, N * sizeof(double));
    if (which == 0) { /* Gx */
        ORC_PAR_FOR
        for (int i2 = 2; i2 < nnx - 1; i2++)
            for (int i1 = 0; i1 < nnz; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                d[id] = ORC_A0 * (f[id] - f[id - nnz]) + ORC_A1 * (f[id + nnz] - f[id - 2 * nnz]);
            }
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1 + (size_t)nnz;
            d[id] = f[id] - f[id - nnz];
            id = (size_t)i1 + (size_t)(nnx - 1) * nnz;
            d[id] = f[id] - f[id - nnz];
        }
    } else if (which == 1) { /* Gz */
        ORC_PAR_FOR
        for (int i2 = 0; i2 < nnx; i2++)
            for (int i1 = 2; i1 < nnz - 1; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                d[id] = ORC_A0 * (f[id] - f[id - 1]) + ORC_A1 * (f[id + 1] - f[id - 2]);
            }
        for (int i2 = 0; i2 < nnx; i2++) {
            size_t id = (size_t)(nnz - 1) + (size_t)i2 * nnz;
            d[id] = f[id] - f[id - 1];
            id = (size_t)1 + (size_t)i2 * nnz;
            d[id] = f[id] - f[id - 1];
        }
    } else if (which == 2) { /* Hx */
        ORC_PAR_FOR
        for (int i2 = 1; i2 < nnx - 2; i2++)
            for (int i1 = 0; i1 < nnz; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                d[id] = ORC_A0 * (f[id + nnz] - f[id]) + ORC_A1 * (f[id + 2 * nnz] - f[id - nnz]);
            }
        for (int i1 = 0; i1 < nnz; i1++) {
            size_t id = (size_t)i1;
            d[id] = f[id + nnz] - f[id];
            id = (size_t)i1 + (size_t)(nnx - 2) * nnz;
            d[id] = f[id + nnz] - f[id];
        }
    } else { /* Hz */
        ORC_PAR_FOR
        for (int i2 = 0; i2 < nnx; i2++)
            for (int i1 = 1; i1 < nnz - 2; i1++) {
                size_t id = (size_t)i1 + (size_t)i2 * nnz;
                d[id] = ORC_A0 * (f[id + 1] - f[id]) + ORC_A1 * (f[id + 2] - f[id - 1]);
            }
        for (int i2 = 0; i2 < nnx; i2++) {
            size_t id = (size_t)(nnz - 2) + (size_t)i2 * nnz;
            d[id] = f[id + 1] - f[id];
            id = (size_t)i2 * nnz;
            d[id] = f[id + 1] - f[id];
        }
    }
}

/* The same four operators and their transposes for the 8th-order operator
 * (dm8_coef / dp8_coef rows, which include the reference's rows at the
 * edges): d = D f, and out += D^T mu as the scatter of each forward row. */
static void op8_apply(int which, const double *f, double *d, int nnz, int nnx) {
#define F8(ix, iz) ((ix) < 0 || (ix) >= nnx || (iz) < 0 || (iz) >= nnz ? 0.0 : f[(size_t)(iz) + (size_t)(ix) * nnz])
    ORC_PAR_FOR
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            float c[4];
            double v = 0.0;
            if (which == 0) { /* Gx = D-x */
                dm8_coef(ix, nnx, c);
                for (int k = 0; k < 4; k++) v += (double)c[k] * (F8(ix + k, iz) - F8(ix - 1 - k, iz));
            } else if (which == 1) { /* Gz = D-z */
                dm8_coef(iz, nnz, c);
                for (int k = 0; k < 4; k++) v += (double)c[k] * (F8(ix, iz + k) - F8(ix, iz - 1 - k));
            } else if (which == 2) { /* Hx = D+x */
                dp8_coef(ix, nnx, c);
                for (int k = 0; k < 4; k++) v += (double)c[k] * (F8(ix + 1 + k, iz) - F8(ix - k, iz));
            } else { /* Hz = D+z */
                dp8_coef(iz, nnz, c);
                for (int k = 0; k < 4; k++) v += (double)c[k] * (F8(ix, iz + 1 + k) - F8(ix, iz - k));
            }
            d[(size_t)iz + (size_t)ix * nnz] = v;
        }
#undef F8
}
static void op8T_add(int which, const double *mu, double *out, int nnz, int nnx) {
#define ADD8(ix, iz, v)                                                          \
    do {                                                                         \
        if ((ix) >= 0 && (ix) < nnx && (iz) >= 0 && (iz) < nnz)                  \
            out[(size_t)(iz) + (size_t)(ix) * nnz] += (v);                       \
    } while (0)
    /* x-direction rows scatter across columns: row blocks in parallel, the
     * columns of a block in order; z-direction rows stay in their column:
     * columns in parallel */
    const int xdir = which == 0 || which == 2;
    const int nblk = xdir ? (nnz + ORC_ROWS - 1) / ORC_ROWS : 1;
    ORC_PAR_FOR
    for (int t = 0; t < (xdir ? nblk : nnx); t++)
    for (int ix = xdir ? 0 : t; ix < (xdir ? nnx : t + 1); ix++)
        for (int iz = xdir ? t * ORC_ROWS : 0; iz < (xdir ? ((t + 1) * ORC_ROWS < nnz ? (t + 1) * ORC_ROWS : nnz) : nnz); iz++) {
            const double m = mu[(size_t)iz + (size_t)ix * nnz];
            float c[4];
            for (int k = 0; k < 4; k++) {
                if (which == 0) {
                    dm8_coef(ix, nnx, c);
                    ADD8(ix + k, iz, c[k] * m);
                    ADD8(ix - 1 - k, iz, -c[k] * m);
                } else if (which == 1) {
                    dm8_coef(iz, nnz, c);
                    ADD8(ix, iz + k, c[k] * m);
                    ADD8(ix, iz - 1 - k, -c[k] * m);
                } else if (which == 2) {
                    dp8_coef(ix, nnx, c);
                    ADD8(ix + 1 + k, iz, c[k] * m);
                    ADD8(ix - k, iz, -c[k] * m);
                } else {
                    dp8_coef(iz, nnz, c);
                    ADD8(ix, iz + 1 + k, c[k] * m);
                    ADD8(ix, iz - k, -c[k] * m);
                }
            }
        }
#undef ADD8
}

/* One forward step of the gradient's FP64 scheme (the stages of f64_step,
 * written with the step's products a, c, g, h kept in the given arrays). */
typedef struct {
    int nnz, nnx, o8, isrc, nts, nw;
    size_t N;
    const float *damp2a, *damp1a, *damp2b, *damp1b;
    const double *kw1, *kw2, *bw1, *bw2, *kappa, *w;
    float fd_dt, dxdz;
    double *px, *pz, *vx, *vz, *p;
} gfwd;

static void gfwd_step(const gfwd *s, int kt, double *a, double *c, double *g, double *h) {
    const int nnz = s->nnz, nnx = s->nnx;
    double *px = s->px, *pz = s->pz, *vx = s->vx, *vz = s->vz, *p = s->p;
    if (s->o8) {
        op8_apply(0, vx, a, nnz, nnx);
        op8_apply(1, vz, c, nnz, nnx);
    } else {
        op_apply(0, vx, a, nnz, nnx);
        op_apply(1, vz, c, nnz, nnx);
    }
    ORC_PAR_FOR
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            px[id] = s->damp2a[ix] * px[id] + s->kw2[id] * a[id];
            pz[id] = s->damp1a[iz] * pz[id] + s->kw1[id] * c[id];
        }
    if (kt <= s->nts)
        px[s->isrc] = px[s->isrc] + s->fd_dt * (kt < s->nw ? s->w[kt] : 0.0) * s->kappa[s->isrc] / (s->dxdz);
    ORC_PAR_FOR
    for (size_t id = 0; id < s->N; id++) p[id] = px[id] + pz[id];
    if (s->o8) {
        op8_apply(2, p, g, nnz, nnx);
        op8_apply(3, p, h, nnz, nnx);
    } else {
        op_apply(2, p, g, nnz, nnx);
        op_apply(3, p, h, nnz, nnx);
    }
    ORC_PAR_FOR
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            vx[id] = s->damp2b[ix] * vx[id] + s->bw2[id] * g[id];
            vz[id] = s->damp1b[iz] * vz[id] + s->bw1[id] * h[id];
        }
}

int orc_gradient(const orc_params *prm, const float *vp, const float *rho,
                 float sx, float sz, int nrec, const float *gx, const float *gz,
                 const double *wavelet, int nwav, const double *adj,
                 double *grad_vp, double *grad_rho,
                 double *grad_kappa, double *grad_bx, double *grad_bz,
                 double *src_adj, double *seis64) {
    return orc_gradient_seg(prm, vp, rho, sx, sz, nrec, gx, gz, wavelet, nwav, adj, grad_vp, grad_rho, grad_kappa,
                            grad_bx, grad_bz, src_adj, seis64, 0);
}

int orc_gradient_seg(const orc_params *prm, const float *vp, const float *rho,
                     float sx, float sz, int nrec, const float *gx, const float *gz,
                     const double *wavelet, int nwav, const double *adj,
                     double *grad_vp, double *grad_rho,
                     double *grad_kappa, double *grad_bx, double *grad_bz,
                     double *src_adj, double *seis64, int segment) {
    if (!prm || !vp || !rho || nrec < 0 || (nrec > 0 && (!gx || !gz))) return -1;
    if (prm->fd_order != 0 && prm->fd_order != 4 && prm->fd_order != 8) return -1;
    const int o8 = prm->fd_order == 8;
    orc_derived d;
    orc_derive(prm, &d);
    if (d.dt_factor < 1 || d.fd_nt < 1) return -2;
    const int nnx = d.nnx, nnz = d.nnz, nb = prm->nb, nt = d.fd_nt;
    const size_t N = (size_t)nnx * nnz;
    float *vel = calloc(N, sizeof(float)), *den = calloc(N, sizeof(float));
    float *bue = calloc(N, sizeof(float)), *bx = calloc(N, sizeof(float)), *bz = calloc(N, sizeof(float));
    double *kappa = calloc(N, sizeof(double));
    expand(vel, vp, nb, nnz, nnx, prm->nz, prm->nx);
    expand(den, rho, nb, nnz, nnx, prm->nz, prm->nx);
    stagger(vel, den, bue, bx, bz, kappa, nnz, nnx);
    if (prm->free_surface) free_surface_rows(kappa, nb, nnz, nnx);
    int nw = wavelet ? nwav : d.nts;
    double *w = calloc((size_t)(nw > 0 ? nw : 0) + 1, sizeof(double));
    if (wavelet) memcpy(w, wavelet, (size_t)nw * sizeof(double));
    else orc_ricker(prm, &d, w);
    float *damp2a = calloc(nnx, 4), *damp2a1 = calloc(nnx, 4), *damp2b = calloc(nnx, 4), *damp2b1 = calloc(nnx, 4);
    float *damp1a = calloc(nnz, 4), *damp1a1 = calloc(nnz, 4), *damp1b = calloc(nnz, 4), *damp1b1 = calloc(nnz, 4);
    sponge_a(0.05f, damp2a, damp2a1, nb, prm->nx);
    sponge_b(0.05f, damp2b, damp2b1, nb, prm->nx);
    sponge_a(0.05f, damp1a, damp1a1, nb, prm->nz);
    sponge_b(0.05f, damp1b, damp1b1, nb, prm->nz);
    int isrc = orc_cell(prm, sx, sz);
    int *gcell = calloc((size_t)nrec + 1, sizeof(int));
    for (int g = 0; g < nrec; g++) gcell[g] = orc_cell(prm, gx[g], gz[g]);
    double *kw1 = malloc(N * 8), *kw2 = malloc(N * 8), *bw1 = malloc(N * 8), *bw2 = malloc(N * 8);
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            kw2[id] = d.dtdx * kappa[id] * damp2a1[ix];
            kw1[id] = d.dtdz * kappa[id] * damp1a1[iz];
            bw2[id] = d.dtdx * bx[id] * damp2b1[ix];
            bw1[id] = d.dtdz * bz[id] * damp1b1[iz];
        }
    const float dxdz = prm->dx * prm->dz;
    /* checkpointing: segments of `seg` steps; the products a, c, g, h of one
     * segment at a time (every step's when there is one segment) and the
     * state at each segment start; a forward alone keeps neither */
    const int seg = segment <= 0 || segment >= nt ? nt : segment;
    const int nseg = (nt + seg - 1) / seg;
    const size_t keep = adj ? (size_t)seg : 1;
    double *A = malloc(N * 8 * keep), *Cc = malloc(N * 8 * keep);
    double *Gg = malloc(N * 8 * keep), *Hh = malloc(N * 8 * keep);
    double *ck = adj && nseg > 1 ? malloc(N * 8 * 4 * (size_t)nseg) : NULL;
    double *px = calloc(N, 8), *pz = calloc(N, 8), *vx = calloc(N, 8), *vz = calloc(N, 8), *p = calloc(N, 8);
    if (!A || !Cc || !Gg || !Hh || (adj && nseg > 1 && !ck)) return -4;
    gfwd fs = {nnz, nnx, o8, isrc, d.nts, nw, N, damp2a, damp1a, damp2b, damp1b, kw1, kw2, bw1, bw2, kappa, w,
               prm->fd_dt, dxdz, px, pz, vx, vz, p};
    /* forward sweep: the state at each segment start, the traces, and the
     * last segment's products */
    for (int j = 0; j < nseg; j++) {
        const int k0 = j * seg, k1 = k0 + seg < nt ? k0 + seg : nt;
        if (ck) {
            double *st = ck + N * 4 * (size_t)j;
            memcpy(st, px, N * 8);
            memcpy(st + N, pz, N * 8);
            memcpy(st + 2 * N, vx, N * 8);
            memcpy(st + 3 * N, vz, N * 8);
        }
        for (int kt = k0; kt < k1; kt++) {
            const size_t sl = adj && j == nseg - 1 ? (size_t)(kt - k0) : 0;
            gfwd_step(&fs, kt, A + N * sl, Cc + N * sl, Gg + N * sl, Hh + N * sl);
            if (seis64 && (kt + 1) % d.dt_factor == 0) {
                int it = (kt + 1) / d.dt_factor - 1;
                if (it < d.real_nt)
                    for (int r = 0; r < nrec; r++) seis64[(size_t)r * d.real_nt + it] = p[gcell[r]];
            }
        }
    }
    /* adjoint, backwards in time */
    double *mpx = calloc(N, 8), *mpz = calloc(N, 8), *mvx = calloc(N, 8), *mvz = calloc(N, 8);
    double *mg = malloc(N * 8), *mh = malloc(N * 8), *q = malloc(N * 8), *mPX = malloc(N * 8), *mPZ = malloc(N * 8);
    double *ma = malloc(N * 8), *mc = malloc(N * 8), *nvx = malloc(N * 8), *nvz = malloc(N * 8);
    double *gk = calloc(N, 8), *gbx = calloc(N, 8), *gbz = calloc(N, 8);
    double gk_src = 0.0;
    if (!adj && src_adj) memset(src_adj, 0, (size_t)nt * sizeof(double));
    for (int j = nseg - 1; j >= 0 && adj; j--) {
        const int k0 = j * seg, k1 = k0 + seg < nt ? k0 + seg : nt;
        if (j < nseg - 1) {
            /* recompute the segment's products from its checkpoint */
            const double *st = ck + N * 4 * (size_t)j;
            memcpy(px, st, N * 8);
            memcpy(pz, st + N, N * 8);
            memcpy(vx, st + 2 * N, N * 8);
            memcpy(vz, st + 3 * N, N * 8);
            for (int kt = k0; kt < k1; kt++) {
                const size_t sl = (size_t)(kt - k0);
                gfwd_step(&fs, kt, A + N * sl, Cc + N * sl, Gg + N * sl, Hh + N * sl);
            }
        }
    for (int kt = k1 - 1; kt >= k0; kt--) {
        double *a = A + N * (size_t)(kt - k0), *c = Cc + N * (size_t)(kt - k0);
        double *g = Gg + N * (size_t)(kt - k0), *h = Hh + N * (size_t)(kt - k0);
        /* vx' = damp2b vx + bw2 g ; vz' = damp1b vz + bw1 h */
        ORC_PAR_FOR
        for (int ix = 0; ix < nnx; ix++)
            for (int iz = 0; iz < nnz; iz++) {
                size_t id = (size_t)iz + (size_t)ix * nnz;
                mg[id] = bw2[id] * mvx[id];
                mh[id] = bw1[id] * mvz[id];
                gbx[id] += d.dtdx * damp2b1[ix] * g[id] * mvx[id];
                gbz[id] += d.dtdz * damp1b1[iz] * h[id] * mvz[id];
                nvx[id] = damp2b[ix] * mvx[id];
                nvz[id] = damp1b[iz] * mvz[id];
            }
        /* g = Hx p', h = Hz p' ; record */
        memset(q, 0, N * 8);
        if (o8) {
            op8T_add(2, mg, q, nnz, nnx);
            op8T_add(3, mh, q, nnz, nnx);
        } else {
            hxT_add(mg, q, nnz, nnx);
            hzT_add(mh, q, nnz, nnx);
        }
        if (adj && (kt + 1) % d.dt_factor == 0) {
            int it = (kt + 1) / d.dt_factor - 1;
            if (it < d.real_nt)
                for (int r = 0; r < nrec; r++) q[gcell[r]] += adj[(size_t)r * d.real_nt + it];
        }
        /* p' = px' + pz' */
        ORC_PAR_FOR
        for (size_t id = 0; id < N; id++) {
            mPX[id] = mpx[id] + q[id];
            mPZ[id] = mpz[id] + q[id];
        }
        /* source term: d/dkappa_src and the injection's transpose */
        if (src_adj) src_adj[kt] = mPX[isrc];
        if (kt <= d.nts) gk_src += mPX[isrc] * (prm->fd_dt * (kt < nw ? w[kt] : 0.0) / (dxdz));
        /* px' = damp2a px + kw2 a ; pz' = damp1a pz + kw1 c */
        ORC_PAR_FOR
        for (int ix = 0; ix < nnx; ix++)
            for (int iz = 0; iz < nnz; iz++) {
                size_t id = (size_t)iz + (size_t)ix * nnz;
                gk[id] += d.dtdx * damp2a1[ix] * a[id] * mPX[id] + d.dtdz * damp1a1[iz] * c[id] * mPZ[id];
                mpx[id] = damp2a[ix] * mPX[id];
                mpz[id] = damp1a[iz] * mPZ[id];
                ma[id] = kw2[id] * mPX[id];
                mc[id] = kw1[id] * mPZ[id];
            }
        /* a = Gx vx, c = Gz vz */
        if (o8) {
            op8T_add(0, ma, nvx, nnz, nnx);
            op8T_add(1, mc, nvz, nnz, nnx);
        } else {
            gxT_add(ma, nvx, nnz, nnx);
            gzT_add(mc, nvz, nnz, nnx);
        }
        memcpy(mvx, nvx, N * 8);
        memcpy(mvz, nvz, N * 8);
    }
    }
    gk[isrc] += gk_src;
    /* with a free surface kappa is held at 0 on rows 0..nb: not a function of
     * vp or rho there */
    if (prm->free_surface)
        for (int ix = 0; ix < nnx; ix++)
            for (int iz = 0; iz <= nb && iz < nnz; iz++) gk[(size_t)iz + (size_t)ix * nnz] = 0.0;
    if (grad_kappa) memcpy(grad_kappa, gk, N * 8);
    if (grad_bx) memcpy(grad_bx, gbx, N * 8);
    if (grad_bz) memcpy(grad_bz, gbz, N * 8);
    /* materials -> buoyancy: bz = 0.5 (b[z] + b[z+1]) (last row 0), bx = 0.5 (b[x] + b[x+1]),
     * bx last column = bz of column nnx-2 (CK:89-119) */
    double *gb = calloc(N, 8);
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz - 1; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            gb[id] += 0.5 * gbz[id];
            gb[id + 1] += 0.5 * gbz[id];
        }
    for (int ix = 0; ix < nnx - 1; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            gb[id] += 0.5 * gbx[id];
            gb[id + nnz] += 0.5 * gbx[id];
        }
    for (int iz = 0; iz < nnz - 1; iz++) {
        size_t last = (size_t)iz + (size_t)(nnx - 1) * nnz, id = (size_t)iz + (size_t)(nnx - 2) * nnz;
        gb[id] += 0.5 * gbx[last];
        gb[id + 1] += 0.5 * gbx[last];
    }
    /* kappa = vp^2 rho, b = 1/rho (rho > 0), then fold the sponge onto the model */
    if (grad_vp) memset(grad_vp, 0, (size_t)prm->nx * prm->nz * 8);
    if (grad_rho) memset(grad_rho, 0, (size_t)prm->nx * prm->nz * 8);
    for (int ix = 0; ix < nnx; ix++)
        for (int iz = 0; iz < nnz; iz++) {
            size_t id = (size_t)iz + (size_t)ix * nnz;
            int mx = ix - nb < 0 ? 0 : (ix - nb > prm->nx - 1 ? prm->nx - 1 : ix - nb);
            int mz = iz - nb < 0 ? 0 : (iz - nb > prm->nz - 1 ? prm->nz - 1 : iz - nb);
            double v = vel[id], r = den[id];
            size_t m = (size_t)mx * prm->nz + mz;
            if (grad_vp) grad_vp[m] += 2.0 * v * r * gk[id];
            if (grad_rho) grad_rho[m] += v * v * gk[id] + (r > 0 ? -gb[id] / (r * r) : 0.0);
        }
    free(gb);
    free(A); free(Cc); free(Gg); free(Hh); free(ck); free(px); free(pz); free(vx); free(vz); free(p);
    free(mpx); free(mpz); free(mvx); free(mvz); free(mg); free(mh); free(q); free(mPX); free(mPZ);
    free(ma); free(mc); free(nvx); free(nvz); free(gk); free(gbx); free(gbz);
    free(kw1); free(kw2); free(bw1); free(bw2); free(gcell); free(w);
    free(vel); free(den); free(bue); free(bx); free(bz); free(kappa);
    free(damp2a); free(damp2a1); free(damp2b); free(damp2b1); free(damp1a); free(damp1a1); free(damp1b); free(damp1b1);
    return 0;
}

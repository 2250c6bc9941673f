/*
 * CPU restatement of SeisAcoMod2D's forward-modelling path (one shot).
 *
 * TEST INFRASTRUCTURE.  This library is the checker for the CUDA product
 * path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * load it.  The product library never links or calls it.
 *
 * Two arithmetic variants of the same scheme:
 *   orc_forward(..., ORC_F64, ...)  the reference's own FP64 wavefields with
 *                                   its float/double mix, operation order kept
 *                                   (src/src_cpu/cpumodelling.cpp,
 *                                    src/src_cpu/cpu_modelling_kernels.cpp);
 *   orc_forward(..., ORC_F32, ...)  the same steps with FP32 wavefields and
 *                                   FP32 per-cell coefficients, the arithmetic
 *                                   the CUDA kernels use (cells where both
 *                                   pressure dampings are 1 carry p = px + pz
 *                                   in px alone).
 * Two options the reference parses and never implements are restated as this
 * project defines them (orc_params.free_surface, orc_params.fd_order = 8); with
 * both at their defaults the oracle is the reference's scheme.
 */
#ifndef S2D_ORACLE_H
#define S2D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_F64 = 64, ORC_F32 = 32 };

typedef struct {
    int nx, nz;        /* physical grid, x-major [nx][nz] */
    int nb;            /* sponge width in cells (reference: npml, cpumodelling.cpp:15) */
    float dx, dz;      /* metres */
    float rec_len;     /* "Time"      seconds */
    float fd_dt;       /* "FD DT"     seconds */
    float real_dt;     /* "DATA DT"   seconds */
    float fm;          /* "Frequency" Hz */
    int free_surface;  /* "Free surface" 1: pressure-release surface at the
                          first model row (kappa = 0 on padded rows 0..nb).
                          The reference parses this key and ignores it
                          (src/src_cpu/json_parser.cpp:236-244); 0 keeps
                          the reference's behaviour. */
    int fd_order;      /* "Order of FD Operator": 0 or 4 the reference's
                          4th-order operator (cpumodelling.cpp:121, NJ == 4);
                          8 the 8th-order staggered operator of this project
                          (the reference runs no step for NJ != 4).
                          orc_gradient handles both. */
} orc_params;

typedef struct {
    int nnx, nnz;      /* padded grid */
    int fd_nt;         /* FD steps            (cpumodelling.cpp:174) */
    int real_nt;       /* recorded samples    (cpumodelling.cpp:175) */
    int dt_factor;     /* FD steps per sample (cpumodelling.cpp:179) */
    int nts;           /* wavelet length      (cpumodelling.cpp:183-188) */
    double dtdx, dtdz; /* (double)(dt * (1/d))  (cpumodelling.cpp:177) */
} orc_derived;

/* Derived run constants exactly as the reference computes them. */
void orc_derive(const orc_params *p, orc_derived *d);

/* Ricker wavelet of length d->nts (cpu_modelling_kernels.cpp:33-62). */
void orc_ricker(const orc_params *p, const orc_derived *d, double *w);

/* Padded cell index of a position in metres (cpumodelling.cpp:284-292,
 * cpu_modelling_kernels.cpp:15-22). */
int orc_cell(const orc_params *p, float x, float z);

/*
 * One shot.  vp, rho: [nx][nz] float32.  Receivers at (gx[g], gz[g]) metres.
 * wavelet: NULL for the reference Ricker, else nwav samples (entries at
 * kt >= nwav count as 0).  kt_stop: number of FD steps to run (<= 0 means
 * the full fd_nt).  seis: [nrec][real_nt] float32, zero-filled beyond the
 * last recorded sample.  state_out (optional): px,pz,vx,vz,p after the last
 * step, 5 arrays of nnx*nnz doubles, x-major.
 * Returns 0 on success, negative on bad arguments.
 */
int orc_forward(const orc_params *p, int precision,
                const float *vp, const float *rho,
                float sx, float sz, int nrec, const float *gx, const float *gz,
                const double *wavelet, int nwav, int kt_stop,
                float *seis, double *state_out);

/*
 * FP64 discrete adjoint of the ORC_F64 forward of one shot (test reference for
 * the CUDA gradient).  adj: the adjoint source dJ/d(seis), [nrec][real_nt]
 * (for the L2 misfit, the residual).  Returns, each optional:
 *   grad_vp, grad_rho  [nx][nz]  dJ/dvp, dJ/drho on the physical grid (the
 *                                 sponge cells fold onto the edge cells they
 *                                 replicate)
 *   grad_kappa, grad_bx, grad_bz [nnx][nnz] dJ/d of the padded materials
 *   src_adj            [fd_nt]   adjoint pressure at the source after each
 *                                 step's source term (the transpose of the
 *                                 injection: d seis / d w is its dot product)
 *   seis64             [nrec][real_nt] the forward traces in double
 */
int orc_gradient(const orc_params *p, const float *vp, const float *rho,
                 float sx, float sz, int nrec, const float *gx, const float *gz,
                 const double *wavelet, int nwav, const double *adj,
                 double *grad_vp, double *grad_rho,
                 double *grad_kappa, double *grad_bx, double *grad_bz,
                 double *src_adj, double *seis64);

/*
 * orc_gradient with checkpointing: the forward keeps its state every
 * `segment` steps and each segment's step products are recomputed from its
 * checkpoint on the way back (segment <= 0 or >= fd_nt: one segment, every
 * product of the run kept).  Bit-identical to orc_gradient for every segment
 * length.  adj == NULL runs the forward alone (seis64) and keeps nothing.
 */
int orc_gradient_seg(const orc_params *p, const float *vp, const float *rho,
                     float sx, float sz, int nrec, const float *gx, const float *gz,
                     const double *wavelet, int nwav, const double *adj,
                     double *grad_vp, double *grad_rho,
                     double *grad_kappa, double *grad_bx, double *grad_bz,
                     double *src_adj, double *seis64, int segment);

/*
 * Threads of orc_gradient / orc_gradient_seg (OpenMP, default 1).  Each
 * parallel loop splits cells whose updates do not depend on one another and
 * keeps the order of the additions into every cell, so the results are the
 * same bits for every thread count.
 */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif

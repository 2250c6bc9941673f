/*
 * seis2d.h -- C ABI of libseis2d, the B200 (sm_100a) implementation of
 * SeisAcoMod2D's forward-modelling hot path: the per-shot 2-D acoustic
 * 4th-order staggered-grid time loop with split-field sponge, Ricker source
 * injection and receiver sampling (and, as options of a model, the
 * free surface and 8th-order operator the reference's job card names but
 * its modelling never implements).
 *
 * Reference seam replaced:
 *   void modelling_module(int my_nsrc, geo2d_t *mygeo2d_sp);
 *   (src/src_cpu/modelling.h:106, defined by every backend:
 *    src/src_cpu/cpumodelling.cpp:158, src/src_gpu/gpumodelling.cu:238)
 * That function takes its inputs from globals (mod_sp, wave_sp, job_sp;
 * src/src_cpu/modelling.h:13-61) and writes the seismogram files itself.
 * Here the same inputs arrive as arguments, the seismograms are returned in
 * caller-owned buffers, and file I/O lives in the host driver entry points at
 * the end of this header (s2d_run_jobcard), which keep the reference's
 * job-card, geometry, model and seismogram formats.
 *
 * Conventions
 *   - Plain C types only; every entry point returns an int status
 *     (S2D_OK = 0, negative = error class) and never aborts the process
 *     (the reference calls MPI::COMM_WORLD.Abort with negative codes).
 *   - The caller owns every buffer it passes.  The library owns the device
 *     memory of a context and frees it in s2d_destroy.
 *   - A context is bound to one CUDA device.  Calls on one context are not
 *     thread-safe; distinct contexts may be used from distinct threads.
 *   - Grids are x-major [nx][nz] with z contiguous, as the reference's model
 *     files and geo2d_t coordinates (metres).
 */
#ifndef SEIS2D_H
#define SEIS2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define S2D_API __attribute__((visibility("default")))
#else
#define S2D_API
#endif

#define S2D_ABI_VERSION 3

/* status codes */
#define S2D_OK 0
#define S2D_ERR_ARG -1      /* bad argument (null pointer, size, id)        */
#define S2D_ERR_CUDA -2     /* CUDA runtime error (text in s2d_last_error)  */
#define S2D_ERR_NOMEM -3    /* device or host allocation failed             */
#define S2D_ERR_GEOM -4     /* source/receiver outside the grid             */
#define S2D_ERR_STATE -5    /* call out of order (e.g. bad continuation)    */
#define S2D_ERR_IO -6       /* file missing, unreadable or of wrong size     */
#define S2D_ERR_JOBCARD -7  /* job card key missing or malformed            */
#define S2D_ERR_STABILITY -8 /* stability / dispersion criterion violated    */
#define S2D_ERR_TIMEOUT -9  /* a bounded device-side wait gave up           */
#define S2D_ERR_NODEV -10   /* no usable CUDA device                         */

/* flags for s2d_forward */
#define S2D_SEIS_DEVICE 0x1u   /* seis_out is a device pointer                 */
#define S2D_PLAIN 0x2u         /* shots one after another (reference order)    */
#define S2D_NO_GRAPH 0x4u      /* launch the time loop step by step            */
#define S2D_SYNC 0x8u          /* return only when device work has finished    */

/* flags for s2d_gradient (with S2D_SEIS_DEVICE for data / seis_out, S2D_NO_GRAPH) */
#define S2D_GRAD_MISFIT 0x10u  /* data is observed seismograms: adjoint source = d - data  */
#define S2D_GRAD_DEVICE 0x20u  /* grad_vp, grad_rho are device pointers                    */

/* flags for s2d_model_create */
#define S2D_MODEL_DEVICE 0x1u  /* vp and rho are device pointers               */
#define S2D_MODEL_FREE_SURFACE 0x2u /* pressure-release surface at the first model
                                   row (job card "Free surface" : "1"), see
                                   s2d_model_create                             */
#define S2D_MODEL_ORDER8 0x4u  /* 8th-order FD operator (job card "Order of FD
                                  Operator" : "8"), see s2d_model_create       */

/* Source/receiver position in metres; layout of crd2d_t
 * (src/src_cpu/modelling.h:35-38). */
typedef struct {
    float x, z;
} s2d_coord;

/* Time-stepping parameters; layout of wave_t (src/src_cpu/modelling.h:27-31):
 * record length "Time", "FD DT", "DATA DT" in seconds, "Frequency" in Hz. */
typedef struct {
    float rec_len, fd_dt, real_dt, dom_freq;
} s2d_wave;

/* One shot: the model it runs on, its source and its receivers.  Replaces one
 * entry of geo2d_t (src/src_cpu/modelling.h:40-45).  rec points to nrec host
 * coordinates. */
typedef struct {
    int model_id;
    s2d_coord src;
    int nrec;
    const s2d_coord *rec;
} s2d_shot;

/* Constants the reference derives from s2d_wave
 * (src/src_cpu/cpumodelling.cpp:168-188). */
typedef struct {
    int fd_nt;     /* FD steps            ceil(Time / FD DT)                 */
    int real_nt;   /* samples per trace   ceil(Time / DATA DT)               */
    int dt_factor; /* FD steps per sample (int)(DATA DT / FD DT)             */
    int nts;       /* Ricker length       (int)(5*sqrt(6)/(pi f)/FD DT) + 1  */
} s2d_steps;

/* Per-call performance record (device time of the time loop). */
typedef struct {
    double loop_ms;          /* CUDA-event time of the FD time loop           */
    double cell_updates;     /* padded cells x steps advanced                 */
    double gcells_per_s;     /* cell_updates / loop_ms                        */
    int kernel_launches;     /* launches of the library's own kernels         */
    int graph_used;          /* 1 if the loop ran as a CUDA graph             */
    int grad_segment;        /* s2d_gradient: checkpoint interval used (steps) */
    int variant, block, stages;  /* launch configuration of the time loop     */
    int seg_len;             /* columns per warp task (first model group)     */
    int autotuned;           /* 1 if this call ran the autotuner's trials     */
    double alg_bytes;        /* s2d_forward: algorithmic DRAM bytes of the loop:
                                44 B per cell and pass over the state, 36 B
                                where both pressure dampings are 1 (the cell
                                carries p alone); a pass is one FD step, or
                                two with the two-step variant                 */
    double sweep_ms;         /* s2d_gradient: CUDA-event time of the forward
                                sweep (checkpoint saves included)              */
    double recompute_ms;     /* s2d_gradient: the recomputes that keep the
                                step products (checkpoint restores included)  */
    double adjoint_ms;       /* s2d_gradient: the adjoint steps; loop_ms minus
                                the three is set-up, adjoint source and
                                finalisation                                   */
    int task_order;          /* task order of the time loop ("task_order")    */
} s2d_stats;

/* ---- library / context ------------------------------------------------ */

/* ABI version of the loaded library (S2D_ABI_VERSION). */
S2D_API int s2d_abi_version(void);

/* Create a context on CUDA device `device`.  No counterpart in the reference
 * (its backends use globals and cudaSetDevice(0), src/src_gpu/gpumodelling.cu:285). */
S2D_API int s2d_create(void **ctx, int device);

/* Free every device buffer and graph of the context. */
S2D_API void s2d_destroy(void *ctx);

/* Text of the last error on this context (never NULL). */
S2D_API const char *s2d_last_error(const void *ctx);

/*
 * Tuning knobs of the step kernel; no counterpart in the reference.  Keys:
 *   "autotune"    1 (default): the first s2d_forward of a batched run of a new
 *                 shape (models, grids, shot counts) with at least 112 steps
 *                 (64 for the 8th-order operator) spends up to 56 (32) of them
 *                 on trials: 9 candidate configurations (variants 4, 16, 15,
 *                 2, 5, 11, 12 in task order 1, and 16 and 15 in task order 0,
 *                 unless "task_order" was set), one untimed and three timed
 *                 launches each, in rounds, then four more timed launches each
 *                 of the two fastest, alternating (the results do not change:
 *                 every candidate computes the same bits); it keeps the fastest
 *                 per FD step for that shape in the context; runs that do not
 *                 tune (shorter calls, S2D_PLAIN) use variant 16.
 *                 0: use "variant", "block" and "stages".
 *                 Setting any of those three turns autotuning off.
 *   "variant"     0 bulk-copy pipeline, 1 plain loads, 2 bulk-copy pipeline
 *                 compiled for 128 registers, 4 plain loads compiled for 128
 *                 registers, 5 two FD steps per launch (the state crosses HBM
 *                 once per two steps; odd step counts end with one one-step
 *                 launch), 11 a CTA of 8 warps on adjacent strips fed by a
 *                 producer warp's 2-D TMA tensor loads through a 4-stage
 *                 shared-memory ring (one block of 288 threads per SM),
 *                 12 the plain-load loop fed by per-lane asynchronous copies
 *                 (cp.async) into a 3-column per-warp ring, 14 variant 4 with
 *                 its column loop unrolled by 4, 15 plain loads with the next
 *                 column's loads issued before the current column is computed
 *                 (3 blocks per SM), 16 the same at 4 blocks per SM (default),
 *                 17 and 18 the prefetch with the loop unrolled by 4 at 4 and
 *                 3 blocks per SM, 20 variant 16's loop in a persistent
 *                 cooperative launch that advances "graph_chunk" steps with a
 *                 bounded grid barrier between steps (an option only: slower
 *                 than per-step launches on the grids measured);
 *                 s2d_gradient always runs one step per launch.
 *                 For batches of S2D_MODEL_ORDER8 models: 7 register windows
 *                 at 3 blocks per SM (default), 8 the same at 2, 9 windows in
 *                 shared memory at 4 (each setting applies to its own order)
 *   "block"       threads per block: 32, 64, 96 or 128 (default 128)
 *   "task_order"  0: consecutive warps take the shots of one tile (the four
 *                 warps of a block share its kappa, bx, bz through L1);
 *                 1: consecutive warps take adjacent strips of one shot (the
 *                 default); setting it keeps the autotuner off this choice
 *   "stages"      bulk-copy ring depth per warp, 2..16 (default 3)
 *   "seg_len"     columns per x-segment of a warp task, 0 = automatic
 *   "spin_limit"  polls of a pipeline barrier before the wait gives up and the
 *                 call returns S2D_ERR_TIMEOUT (default 2^20)
 *   "fast_rows"   1 (default): strips clear of the z-sponge and the edge rows
 *                 use literal row coefficients; 0: every strip reads them
 *                 (same results, a check of the fast path)
 *   "graph_chunk" FD steps per captured CUDA graph, replayed as often as a
 *                 run needs (default 64)
 *   "adjoint8_form" s2d_gradient of 8th-order models: 0 (default) one
 *                 streaming pass per step (8-column shared-memory rings for the
 *                 x-gathers, shuffles for the z-gathers), 1 two cell-parallel
 *                 passes with the gathers read from memory
 *   "products_variant" s2d_gradient's forward recompute that keeps the step
 *                 derivatives: 3 plain loads, 19 plain loads with the next
 *                 column prefetched (default)
 *   "adjoint_blocks" s2d_gradient adjoint kernel built for 2, 3 or 4 blocks
 *                 of 128 threads per SM, or 12: 2 blocks per SM with the next
 *                 column's loads issued before a column is computed, or
 *                 13 (default) / 14: 3 / 2 blocks per SM with the column
 *                 inputs copied into shared memory (cp.async) 1 / 2 columns
 *                 ahead, or 15: 3 blocks per SM with the per-shot inputs
 *                 copied 2 columns ahead; every form computes the same bits
 *   "grad_segment" s2d_gradient checkpoint interval in FD steps, 0 = the
 *                 longest that fits in free device memory (default)
 *   "inject_wait_fault"  test knob: >= 0 makes every warp skip the copies of
 *                 that pipeline iteration of its first task (bulk-copy and TMA
 *                 kernels), or block 0 skip its arrival at the grid barrier
 *                 after that step (persistent kernel), so a bounded wait runs
 *                 out (no fault, no hang); -1 (default) disables
 * Options apply to the next s2d_forward call.
 */
S2D_API int s2d_set_option(void *ctx, const char *key, long value);

/* Derived step counts for a wave description, host-only, no device needed
 * (src/src_cpu/cpumodelling.cpp:174-188). */
S2D_API int s2d_derive_steps(const s2d_wave *wave, s2d_steps *out);

/* ---- models -------------------------------------------------------------- */

/*
 * Upload a model: nx*nz vp (m/s) and rho (kg/m^3), x-major, grid spacing
 * dx, dz (m) and sponge width nb cells on each side (the reference fixes
 * nb = 32, src/src_cpu/cpumodelling.cpp:15).  The library expands it into the
 * sponge by edge replication (cpumodelling.cpp:39-60) and forms
 * kappa = vp^2 rho and the staggered buoyancies (cpu_modelling_kernels.cpp:
 * 64-121) on the device.  Returns a model id in *model_id.
 *
 * S2D_MODEL_FREE_SURFACE: the first model row (padded row nb) becomes a
 * pressure-release surface in its vacuum form: kappa is held at 0 on padded
 * rows 0..nb, so p = 0 on the surface row and above it, a source on those rows
 * injects nothing (its amplitude scales with kappa at the source), receivers
 * there record 0, and s2d_gradient treats kappa on those rows as fixed.  The
 * step kernels are unchanged.  The reference parses the job card's
 * "Free surface" key and ignores it (src/src_cpu/json_parser.cpp:236-244; its
 * Instructions file: "Free surface yet not implemented"), so without this
 * flag the results are the reference's.
 *
 * S2D_MODEL_ORDER8: shots on this model run the staggered 8th-order operator
 * D- f[i] = sum_k c_k (f[i+k-1] - f[i-k]), D+ f[i] = sum_k c_k (f[i+k] - f[i-k+1]),
 * c = (1225/1024, -245/3072, 49/5120, -5/7168) in float, with the reference's
 * 4th-order pair, plain difference and zero row where the 8 taps would leave
 * the grid; sponge, source and receivers as for order 4.  The reference
 * parses "Order of FD Operator" and steps only for 4 (cpumodelling.cpp:121).
 * All shots of one s2d_forward call must share the order; s2d_gradient
 * returns the gradient of the 8th-order scheme for order-8 models.  Stable
 * for vmax dt / min(dx, dz) <= 0.549 (0.606 for order 4).
 */
S2D_API int s2d_model_create(void *ctx, int nx, int nz, float dx, float dz, int nb,
                     const float *vp, const float *rho, unsigned flags, int *model_id);

/* Release a model's device memory. */
S2D_API int s2d_model_destroy(void *ctx, int model_id);

/* ---- forward modelling ---------------------------------------------------- */

/*
 * Run the FD time loop for `nshots` shots (the loop of
 * src/src_cpu/cpumodelling.cpp:326-380 with FDOperator_4 at :115-156).
 *
 *   wave        time stepping; every shot uses the same one
 *   wavelet     NULL for the reference Ricker (cpu_modelling_kernels.cpp:33-62),
 *               else nwavelet source samples, one per FD step (missing
 *               samples count as 0)
 *   kt_begin    0 starts all shots from rest; > 0 continues the previous
 *               call's shots from that FD step (must equal where it stopped)
 *   kt_count    FD steps to run in this call; <= 0 runs to the end (fd_nt)
 *   seis_out    nshots consecutive blocks, block s is [nrec_s][real_nt]
 *               float32 (sample fastest) -- the reference's output file
 *               layout (cpumodelling.cpp:367-374).  Samples recorded in this
 *               call's step range are written; others are left as they are.
 *   flags       S2D_SEIS_DEVICE, S2D_PLAIN, S2D_NO_GRAPH, S2D_SYNC
 *   stats       optional, filled with the device time of the loop
 *
 * Without S2D_PLAIN all shots advance together, one launch per FD step
 * covering every shot (models of different sizes included), captured as a
 * CUDA graph.  With S2D_PLAIN each shot runs its whole loop before the next
 * starts, as the reference does.  Each shot starts from a zero wavefield (the
 * reference zeroes only the first nnz cells between shots of one rank,
 * cpumodelling.cpp:343-348; its first shot per rank is the behaviour kept).
 */
S2D_API int s2d_forward(void *ctx, const s2d_shot *shots, int nshots, const s2d_wave *wave,
                const double *wavelet, int nwavelet, int kt_begin, int kt_count,
                float *seis_out, unsigned flags, s2d_stats *stats);

/* ---- FWI gradient ----------------------------------------------------------------- */

/*
 * Gradient of a seismogram objective with respect to vp and rho of one model,
 * summed over `nshots` shots that all use that model.  No counterpart in the
 * reference (its job_t::adj flag is declared and never used,
 * src/src_cpu/modelling.h:51).  It is the exact discrete adjoint of the FP32
 * forward of s2d_forward: a forward sweep saving the wavefields every
 * `grad_segment` steps, then, segment by segment backwards, a forward
 * recompute that keeps the step derivatives and the adjoint time steps
 * (transposed 4th-order operators, sponge and edge rows included) with the
 * imaging terms for kappa = vp^2 rho, the staggered buoyancies and the
 * kappa-scaled source; the chain rule to vp, rho and the fold of the sponge onto
 * the model edge cells it replicates finish it.
 *
 *   data      without S2D_GRAD_MISFIT: dJ/d(seis), the adjoint source, same
 *             layout as s2d_forward's seis_out (nshots blocks [nrec][real_nt]);
 *             with S2D_GRAD_MISFIT: observed seismograms, J = 0.5 ||d - data||^2
 *   grad_vp, grad_rho   [nx][nz] of the model, overwritten
 *   seis_out  optional: the forward seismograms
 *   misfit    optional: J (S2D_GRAD_MISFIT)
 *   grad_wavelet  optional host array [nshots][fd_nt]: dJ/dw[kt], the gradient
 *             with respect to the source samples (0 where no sample is injected)
 *   flags     S2D_GRAD_MISFIT, S2D_GRAD_DEVICE, S2D_SEIS_DEVICE, S2D_NO_GRAPH
 */
S2D_API int s2d_gradient(void *ctx, const s2d_shot *shots, int nshots, const s2d_wave *wave,
                         const double *wavelet, int nwavelet, const float *data,
                         float *grad_vp, float *grad_rho, float *seis_out, double *misfit,
                         double *grad_wavelet, unsigned flags, s2d_stats *stats);

/* ---- host driver: the reference's files ----------------------------------------- */

/* Parsed job card: the fields of mod_t, wave_t and job_t the reference fills
 * from it (src/src_cpu/modelling.h:13-61, json_parser.cpp:122-300). */
typedef struct {
    char velfile[224], densfile[224];
    int nx, nz;
    float dx, dz;
    s2d_wave wave;
    int geomflag;          /* 0: explicit geometry file, 1: shot file */
    int frsf;              /* "Free surface": 1 models with S2D_MODEL_FREE_SURFACE (the
                              reference parses the key and ignores it) */
    int fdop;              /* FD order (only 4 exists) */
    char jbtype[8];        /* "New" or "Restart" */
    char shotfile[224], geomfile[224];
    char jobname[256];     /* card basename without extension + "_" */
    char tmppath[512];     /* output directory, with trailing '/' */
} s2d_jobcard;

/* Source/receiver geometry of all shots (geo2d_t, src/src_cpu/modelling.h:40-45). */
typedef struct {
    int nsrc;
    int *nrec;             /* [nsrc] */
    s2d_coord *src;        /* [nsrc] */
    s2d_coord **rec;       /* [nsrc][nrec[s]] */
} s2d_geometry;

/* Read a job card (json_parser.cpp:13-300).  Host only.  On failure errbuf
 * (errlen bytes, optional) names the problem and the reference's abort code. */
S2D_API int s2d_jobcard_read(const char *path, s2d_jobcard *out, char *errbuf, size_t errlen);

/* Build the geometry the card names: shot file with split / end-on-left /
 * end-on-right spreads (create_geometry.cpp:15-444) or explicit sx,sz,gx,gz
 * file (read_receiver.cpp:14-306).  Host only.  Free with s2d_geometry_free. */
S2D_API int s2d_geometry_read(const s2d_jobcard *job, s2d_geometry *out, char *errbuf, size_t errlen);
S2D_API void s2d_geometry_free(s2d_geometry *geometry);

/* Stability (dt <= 0.606 h_min / v_max) and dispersion (2 f <= v_min / (5 h_max))
 * criteria of check_stability.cpp:8-72.  Host only.  For job->fdop == 8 the
 * stability bound is 0.549 h_min / v_max (the 8th-order operator; no
 * counterpart in the reference). */
S2D_API int s2d_check_stability(const s2d_jobcard *job, float vmin, float vmax, char *errbuf, size_t errlen);

/*
 * Run the whole job of a card on `device`: read card, geometry and models
 * (model.cpp:12-64), check stability (skipped when check_stability == 0),
 * model every shot (batched, as many per launch as fit in device memory) and
 * write each seismogram, [nrec][real_nt] float32.  Replaces Modelling_master +
 * modelling_module (modelling_master.cpp:10-92, cpumodelling.cpp:158-383).
 *   nb      sponge width (32 in the reference)
 *   naming  0: <outdir>/<jobname>seismogram.bin, the CPU backend's single file
 *              (cpumodelling.cpp:370-374; every shot writes it, the last wins)
 *           1: <outdir>/<jobname>sx<%.2f>_seismogram.bin per shot, the CUDA
 *              backend's names (gpumodelling.cu:471-477)
 * "Job type" Restart skips the shots before the index in
 * <outdir>/<jobname>checkpoint_rank0.txt (cpumodelling.cpp:294-321); unlike
 * the reference, this driver writes that file after every completed shot.
 */
S2D_API int s2d_run_jobcard(const char *jobcard_path, int device, int nb, int naming,
                            int check_stability, int verbose, char *errbuf, size_t errlen);

/*
 * Shots of rank `rank` of `nranks`: the contiguous block [*start, *start +
 * *count) of nsrc, the first nsrc % nranks ranks one shot longer, as
 * calculate_workload assigns them (workload.cpp:12-62).  S2D_ERR_ARG when
 * nsrc < nranks (the reference aborts with -8) or the rank is out of range.
 * Host only.
 */
S2D_API int s2d_workload(int nsrc, int nranks, int rank, int *start, int *count);

/*
 * s2d_run_jobcard for one rank of a multi-process job (one process per GPU,
 * replacing the MPI master/worker split of modelling_master.cpp /
 * modelling_worker.cpp and the per-device OpenMP team of
 * gpumodelling_multi.cu:292-420): models the rank's block of shots
 * (s2d_workload) and keeps the restart index of the block, counted from its
 * first shot, in <outdir>/<jobname>checkpoint_rank<rank>.txt as the reference
 * does (cpumodelling.cpp:294-321).  Output files are named by the shot's
 * place in the whole geometry.  s2d_run_jobcard is rank 0 of 1.
 */
S2D_API int s2d_run_jobcard_rank(const char *jobcard_path, int device, int nb, int naming,
                                 int check_stability, int verbose, int rank, int nranks,
                                 char *errbuf, size_t errlen);

/* ---- forward modelling without device allocation ----------------------------- */

/* Size of the device scratch s2d_forward_static works in (32 MiB). */
#define S2D_STATIC_SCRATCH_BYTES (32u << 20)

/* flags for s2d_forward_static (bits of their own: no other flag of this
 * header is accepted there) */
#define S2D_STATIC_MODEL_DEVICE 0x100u /* vp and rho are device pointers       */
#define S2D_STATIC_SEIS_DEVICE 0x200u  /* seis_out is a device pointer         */

/*
 * One shot of forward modelling that allocates no device memory.  No
 * counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc when they want a shot modelled: a
 * service that reserves its device memory at start-up and forbids allocation
 * afterwards, a program whose own allocator already holds the device memory,
 * or a latency-critical loop that cannot afford the device-wide
 * synchronisation cudaMalloc/cudaFree cause.  The wavefields, materials,
 * tables and staging copies live in a static device array of
 * S2D_STATIC_SCRATCH_BYTES that every GPU loading this library holds until the
 * process exits -- enough for a padded grid of roughly 800 x 800 cells.  A job
 * that needs more returns S2D_ERR_NOMEM with the size it needs in errbuf.
 *
 * Same scheme, numbers and output layout as s2d_forward for one shot with the
 * reference Ricker wavelet and the reference's 4th-order operator without a
 * free surface: model [nx][nz] (vp, rho), sponge width nb, wave, shot->src and
 * shot->rec (shot->model_id is ignored), seis_out [nrec][real_nt].  flags:
 * S2D_STATIC_MODEL_DEVICE (vp, rho are device pointers) and
 * S2D_STATIC_SEIS_DEVICE (seis_out is a device pointer), independently;
 * otherwise host pointers.  Any other bit (S2D_MODEL_FREE_SURFACE and
 * S2D_MODEL_ORDER8 included: this entry has neither option) returns
 * S2D_ERR_ARG.  stream: a cudaStream_t, NULL for the legacy default stream;
 * the call returns when the shot is done.  A failed device self-check (builds
 * with S2D_DEVICE_CHECKS) returns S2D_ERR_CUDA.  errbuf (optional, errlen
 * bytes) receives a message on failure.
 *
 * Every call on a device shares the one scratch array, which keeps the last
 * call's contents; each call clears what must start at zero.  Calls whose
 * device work overlaps on one GPU (several threads or streams at once) race
 * on the array: serialise them.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress, with that device current)
 * and may load the library's device code; make it before starting any stream
 * capture on that device.
 */
S2D_API int s2d_forward_static(int device, int nx, int nz, float dx, float dz, int nb,
                               const float *vp, const float *rho, const s2d_wave *wave,
                               const s2d_shot *shot, float *seis_out, unsigned flags,
                               void *stream, char *errbuf, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* SEIS2D_H */

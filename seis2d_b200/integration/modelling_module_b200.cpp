// modelling_module() for SeisAcoMod2D's host program, on libseis2d.
//
// The reference picks its modelling backend at link time: every backend
// defines `void modelling_module(int my_nsrc, geo2d_t *mygeo2d_sp)`
// (src/src_cpu/modelling.h:106), and Modelling_master / Modelling_worker call
// it once per rank with the rank's shots (modelling_master.cpp:85,
// modelling_worker.cpp:67).  This file is that function for B200: link it,
// with libseis2d, in place of cpumodelling.o.  It takes its inputs from the
// reference's globals (mod_sp, wave_sp, job_sp; modelling.h:13-61) and
// behaves as the CPU backend does (cpumodelling.cpp:158-383):
//   * "Job type" New starts at the rank's first shot; Restart reads the index
//     to start from in <tmppath><jobname>checkpoint_rank<rank>.txt (abort -10
//     when it is missing, -11 for any other job type);
//   * each shot's seismogram, [nrec][real_nt] float32, is written to
//     <tmppath><jobname>seismogram.bin (every shot writes the same file, the
//     last one wins, as in the reference);
//   * errors abort the MPI job with a negative code (-20 here: libseis2d
//     failed; its message goes to stderr).
// Differences: the sponge is 32 cells (the reference's npml) unless the
// environment sets S2D_NB; the GPU is the rank's local one (S2D_DEVICE, else
// 0); each shot starts from a zero wavefield; the rank's shots run batched,
// as many per launch sequence as fit in device memory.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mpi.h"
#include "modelling.h"
#include "seis2d.h"

namespace {

int env_int(const char *name, int dflt) {
    const char *v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

void die(void *ctx, const char *what) {
    std::fprintf(stderr, "\n libseis2d: %s: %s\n", what, ctx ? s2d_last_error(ctx) : "no context");
    MPI::COMM_WORLD.Abort(-20);
}

}  // namespace

void modelling_module(int my_nsrc, geo2d_t *g) {
    const int rank = MPI::COMM_WORLD.Get_rank();
    const int nb = env_int("S2D_NB", 32);
    void *ctx = nullptr;
    if (s2d_create(&ctx, env_int("S2D_DEVICE", 0)) != S2D_OK) die(nullptr, "no usable CUDA device");

    // mod_sp->vel2d / rho2d are nx rows of nz floats (model.cpp:12-44)
    const int nx = mod_sp->nx, nz = mod_sp->nz;
    std::vector<float> vp((size_t)nx * nz), rho((size_t)nx * nz);
    for (int ix = 0; ix < nx; ++ix) {
        std::memcpy(&vp[(size_t)ix * nz], mod_sp->vel2d[ix], sizeof(float) * nz);
        std::memcpy(&rho[(size_t)ix * nz], mod_sp->rho2d[ix], sizeof(float) * nz);
    }
    int model = 0;
    // job_sp->frsf ("Free surface", json_parser.cpp:236-244) is parsed and
    // ignored by the reference's modelling; here 1 gives a pressure-release
    // surface at the first model row
    // job_sp->fdop ("Order of FD Operator"): the reference steps only for 4
    // (cpumodelling.cpp:121) and writes zero traces otherwise; here 8 runs the
    // 8th-order operator and other values stop the job
    if (job_sp->fdop != 4 && job_sp->fdop != 8) die(ctx, "Order of FD Operator must be 4 or 8");
    const unsigned mflags = (job_sp->frsf ? S2D_MODEL_FREE_SURFACE : 0u) | (job_sp->fdop == 8 ? S2D_MODEL_ORDER8 : 0u);
    if (s2d_model_create(ctx, nx, nz, mod_sp->dx, mod_sp->dz, nb, vp.data(), rho.data(), mflags, &model) != S2D_OK)
        die(ctx, "model");

    s2d_wave w;  // the fields of wave_t (modelling.h:27-31)
    w.rec_len = wave_sp->rec_len;
    w.fd_dt = wave_sp->fd_dt_sec;
    w.real_dt = wave_sp->real_dt_sec;
    w.dom_freq = wave_sp->dom_freq;
    s2d_steps st;
    if (s2d_derive_steps(&w, &st) != S2D_OK) die(ctx, "time stepping");

    // New / Restart (cpumodelling.cpp:294-321)
    const std::string log = std::string(job_sp->tmppath) + job_sp->jobname + "checkpoint_rank" +
                            std::to_string(rank) + ".txt";
    int istart = 0;
    if (std::strcmp(job_sp->jbtype, "Restart") == 0) {
        FILE *f = std::fopen(log.c_str(), "r");
        if (!f) {
            std::fprintf(stderr, "\n Rank: %d   Error !!! in opening log file: %s", rank, log.c_str());
            MPI::COMM_WORLD.Abort(-10);
        }
        if (std::fscanf(f, "%d", &istart) != 1) istart = 0;
        std::fclose(f);
    } else if (std::strcmp(job_sp->jbtype, "New") != 0) {
        std::fprintf(stderr, "\n Error !!! Rank: %d   Unknown job status", rank);
        MPI::COMM_WORLD.Abort(-11);
    }
    std::printf("\n Rank: %d   Started Modelling.......", rank);

    const std::string seis_file = std::string(job_sp->tmppath) + job_sp->jobname + "seismogram.bin";
    int batch = my_nsrc > istart ? my_nsrc - istart : 1;
    for (int s0 = istart; s0 < my_nsrc;) {
        const int n = batch < my_nsrc - s0 ? batch : my_nsrc - s0;
        std::vector<s2d_shot> shots(n);
        size_t total = 0;
        for (int k = 0; k < n; ++k) {
            shots[k].model_id = model;
            shots[k].src.x = g->src2d_sp[s0 + k].x;  // crd2d_t has the layout of s2d_coord
            shots[k].src.z = g->src2d_sp[s0 + k].z;
            shots[k].nrec = g->nrec[s0 + k];
            shots[k].rec = reinterpret_cast<const s2d_coord *>(g->rec2d_sp[s0 + k]);
            total += (size_t)g->nrec[s0 + k] * st.real_nt;
        }
        std::vector<float> seis(total);
        const int e = s2d_forward(ctx, shots.data(), n, &w, nullptr, 0, 0, 0, seis.data(), 0, nullptr);
        if (e == S2D_ERR_NOMEM && n > 1) {  // fewer shots per launch sequence
            batch = n / 2;
            continue;
        }
        if (e != S2D_OK) die(ctx, "forward modelling");
        size_t off = 0;
        for (int k = 0; k < n; ++k) {
            const size_t cnt = (size_t)g->nrec[s0 + k] * st.real_nt;
            FILE *f = std::fopen(seis_file.c_str(), "wb");
            if (!f) die(ctx, "cannot write the seismogram file");
            std::fwrite(seis.data() + off, sizeof(float), cnt, f);
            std::fclose(f);
            off += cnt;
            std::printf("\n Rank: %d   Shot remaining: %d", rank, my_nsrc - (s0 + k + 1));
        }
        s0 += n;
    }
    std::printf("\n Rank: %d   Finished Modelling.......\n", rank);
    s2d_destroy(ctx);
}

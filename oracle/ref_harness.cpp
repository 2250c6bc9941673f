/*
 * Harness main for the reference CPU oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * It links the reference's own, unmodified src/src_cpu objects (built by
 * oracle/Makefile from the read-only reference tree into oracle/_ref/) and
 * performs the steps of Modelling_master (src/src_cpu/modelling_master.cpp:
 * 18-62) for a single rank:
 *   set_job_name -> read_json_objects -> set_json_object -> geometry
 *   (read_recv2d | read_source2d) -> print_single_source_geometry ->
 *   calculate_workload/master_workload -> read2d x2 -> minmax2d ->
 *   check_stability -> modelling_module.
 * Switches, all off by default:
 *   --no-stability  skip check_stability() (a diagnostic that aborts on
 *                   grids such as the 3201x1201 / 7.62 m / 20 Hz case whose
 *                   dispersion criterion fails by 2%);
 *   --time          print the wall time of modelling_module() as
 *                   "ORACLE_TIME <seconds>" on its own line;
 *   --dump-job FILE stop after the geometry is built (no model files are
 *                   read) and write the parsed job card (mod_t, wave_t,
 *                   job_t fields) and every shot's source and receivers, as
 *                   the reference holds them, to FILE;
 *   --check VMIN VMAX  with --dump-job: then run check_stability() with
 *                   those velocity bounds (it exits with the reference's
 *                   abort code when a criterion fails) and append "STABLE".
 * The reference's main() (src/src_cpu/main.cpp:52) is compiled with
 * -Dmain=seisacomod2d_reference_main so that its globals (mod_sp, wave_sp,
 * geo2d_sp, job_sp; main.cpp:47-50) are the ones used here.
 */
#include "mpi.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include "modelling.h"

int main(int argc, char **argv) {
    bool stability = true, timeit = false, check = false;
    char *job = nullptr, *dump = nullptr;
    float cvmin = 0, cvmax = 0;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--no-stability")) stability = false;
        else if (!std::strcmp(argv[i], "--time")) timeit = true;
        else if (!std::strcmp(argv[i], "--dump-job") && i + 1 < argc) dump = argv[++i];
        else if (!std::strcmp(argv[i], "--check") && i + 2 < argc) {
            check = true;
            cvmin = (float)std::atof(argv[++i]);
            cvmax = (float)std::atof(argv[++i]);
        } else job = argv[i];
    }
    if (!job) {
        std::fprintf(stderr, "usage: %s [--no-stability] [--time] <jobcard>\n", argv[0]);
        return 2;
    }
    MPI::Init(argc, argv);

    map<string, string> map_json;
    set_job_name(job);
    read_json_objects(job, map_json);
    set_json_object(map_json);
    if (job_sp->geomflag == 0) read_recv2d(job_sp->geomfile);
    else read_source2d(job_sp->shotfile);
    print_single_source_geometry();
    if (dump) {
        FILE *f = std::fopen(dump, "w");
        if (!f) return 3;
        std::fprintf(f, "velfile %s\ndensfile %s\nnx %d\nnz %d\ndx %.9g\ndz %.9g\n", mod_sp->velfile,
                     mod_sp->densfile, mod_sp->nx, mod_sp->nz, mod_sp->dx, mod_sp->dz);
        std::fprintf(f, "rec_len %.9g\nfd_dt %.9g\nreal_dt %.9g\ndom_freq %.9g\n", wave_sp->rec_len,
                     wave_sp->fd_dt_sec, wave_sp->real_dt_sec, wave_sp->dom_freq);
        std::fprintf(f, "geomflag %d\nfdop %d\nfrsf %d\njbtype %s\njobname %s\ntmppath %s\n", job_sp->geomflag,
                     job_sp->fdop, job_sp->frsf, job_sp->jbtype, job_sp->jobname, job_sp->tmppath);
        std::fprintf(f, "nsrc %d\n", geo2d_sp->nsrc);
        for (int s = 0; s < geo2d_sp->nsrc; ++s) {
            std::fprintf(f, "shot %d %.9g %.9g %d\n", s, geo2d_sp->src2d_sp[s].x, geo2d_sp->src2d_sp[s].z,
                         geo2d_sp->nrec[s]);
            for (int g = 0; g < geo2d_sp->nrec[s]; ++g)
                std::fprintf(f, "%.9g %.9g\n", geo2d_sp->rec2d_sp[s][g].x, geo2d_sp->rec2d_sp[s][g].z);
        }
        std::fclose(f);
        if (check) {
            mod_sp->vmin = cvmin;
            mod_sp->vmax = cvmax;
            check_stability();
            f = std::fopen(dump, "a");
            if (!f) return 3;
            std::fprintf(f, "STABLE\n");
            std::fclose(f);
        }
        return 0;
    }

    wrkld_t *wrkld_sp = new wrkld_t[1];
    geo2d_t *mygeo2d_sp = new geo2d_t[1];
    calculate_workload(geo2d_sp->nsrc, wrkld_sp);
    int my_nsrc = wrkld_sp[0].myNsrc;
    mygeo2d_sp->nrec = new int[my_nsrc];
    mygeo2d_sp->src2d_sp = new crd2d_t[my_nsrc];
    mygeo2d_sp->rec2d_sp = new crd2d_t *[my_nsrc];
    send_workload(wrkld_sp);
    master_workload(wrkld_sp, mygeo2d_sp);

    mod_sp->vel2d = new float *[mod_sp->nx];
    mod_sp->rho2d = new float *[mod_sp->nx];
    for (int ix = 0; ix < mod_sp->nx; ix++) {
        mod_sp->vel2d[ix] = new float[mod_sp->nz];
        mod_sp->rho2d[ix] = new float[mod_sp->nz];
    }
    read2d(mod_sp->velfile, mod_sp->vel2d, mod_sp->nx, mod_sp->nz);
    read2d(mod_sp->densfile, mod_sp->rho2d, mod_sp->nx, mod_sp->nz);
    minmax2d(mod_sp->vel2d, mod_sp->nx, mod_sp->nz, mod_sp->vmin, mod_sp->vmax);
    if (stability) check_stability();

    double t0 = MPI::Wtime();
    modelling_module(my_nsrc, mygeo2d_sp);
    double t1 = MPI::Wtime();
    std::fflush(stdout);
    if (timeit) std::printf("\nORACLE_TIME %.6f\n", t1 - t0);
    std::printf("\n");
    return 0;
}

// seis2d_run: the reference program's command line on libseis2d.
//
//   seis2d_run [--device D] [--nb N] [--naming cpu|gpu] [--no-stability] [--quiet] <jobcard>
//
// Same job card, geometry, model and seismogram files as
// `mpirun -np 1 SeisAcoMod2D_*.exe <jobcard>` (Instructions:81-88); the
// modelling runs on one B200.  Exit status 0 on success, 1 on any error
// (the message names the reference's abort code where it has one).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "seis2d.h"

int main(int argc, char **argv) {
    int device = 0, nb = 32, naming = 0, stab = 1, verbose = 1;
    const char *card = nullptr;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--nb") && i + 1 < argc) nb = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--naming") && i + 1 < argc) naming = !std::strcmp(argv[++i], "gpu");
        else if (!std::strcmp(argv[i], "--no-stability")) stab = 0;
        else if (!std::strcmp(argv[i], "--quiet")) verbose = 0;
        else card = argv[i];
    }
    if (!card) {
        std::fprintf(stderr, "usage: %s [--device D] [--nb N] [--naming cpu|gpu] [--no-stability] [--quiet] <jobcard>\n",
                     argv[0]);
        return 2;
    }
    char err[1024] = {0};
    const int rc = s2d_run_jobcard(card, device, nb, naming, stab, verbose, err, sizeof err);
    if (rc != S2D_OK) {
        std::fprintf(stderr, "seis2d_run: error %d: %s\n", rc, err);
        return 1;
    }
    return 0;
}

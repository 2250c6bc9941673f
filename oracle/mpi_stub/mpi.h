/*
 * Single-rank stand-in for the MPI C++ bindings used by the reference CPU
 * host program (src/src_cpu/*.cpp of SeisAcoMod2D).  TEST INFRASTRUCTURE:
 * this header exists only so that the reference's own CPU sources compile
 * unmodified into the oracle binary under oracle/_ref/.  Nothing in the
 * product links against it.
 *
 * Semantics: one rank (rank 0, size 1); Send/Recv are never reached with
 * size 1 (workload.cpp:52-60 only sends to ranks >= 1); Abort(code) prints
 * the code and exits the process with it, as MPI_Abort would for one rank.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/time.h>
#include <unistd.h>

typedef int MPI_Datatype;
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_FLOAT 3

namespace MPI {

class Comm {
public:
    int Get_rank() const { return 0; }
    int Get_size() const { return 1; }
    void Abort(int code) const {
        std::fprintf(stderr, "\n[mpi-stub] Abort(%d)\n", code);
        std::fflush(stdout);
        std::fflush(stderr);
        std::exit(code & 0xff);
    }
    void Send(const void *, int, MPI_Datatype, int, int) const {
        std::fprintf(stderr, "\n[mpi-stub] Send reached with one rank\n");
        std::exit(99);
    }
    void Recv(void *, int, MPI_Datatype, int, int) const {
        std::fprintf(stderr, "\n[mpi-stub] Recv reached with one rank\n");
        std::exit(99);
    }
};

static const Comm COMM_WORLD;

inline void Init(int &, char **&) {}

inline double Wtime() {
    struct timeval tv;
    gettimeofday(&tv, 0);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

inline void Get_processor_name(char *name, int &len) {
    std::strcpy(name, "oracle");
    len = 6;
}

}  // namespace MPI

inline int MPI_Finalize() { return 0; }

#endif

// Host-side set-up quantities of one run, computed with the reference's
// float/double rules so that the device sees the same coefficients the
// reference CPU path uses.
#pragma once

#include <vector>

#include "../../include/seis2d.h"

namespace s2d {

struct RunSteps {
    int fd_nt, real_nt, dt_factor, nts;
    double dtdx, dtdz;
};

// cpumodelling.cpp:168-188
RunSteps derive_steps(const s2d_wave &w, float dx, float dz);

// cpu_modelling_kernels.cpp:33-62 (iss = 2): nts samples.
std::vector<double> ricker(const s2d_wave &w, int nts);

// Sponge profiles of one axis with n physical cells and width nb:
//   a  = integer nodes  (cpu_modelling_kernels.cpp:123-153)
//   b  = half nodes     (cpu_modelling_kernels.cpp:155-199)
// damp is the multiplicative taper, damp1 its square root (exp(-x^2/2)).
void sponge_a(int nb, int n, std::vector<float> &damp, std::vector<float> &damp1);
void sponge_b(int nb, int n, std::vector<float> &damp, std::vector<float> &damp1);

// Padded cell coordinates of a position in metres: (int)(x * (1.0f/dx)) + nb
// (cpumodelling.cpp:288-289, cpu_modelling_kernels.cpp:15-22).
void cell_of(float x, float z, float dx, float dz, int nb, int &ix, int &iz);

}  // namespace s2d

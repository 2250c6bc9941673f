// Reference-exact host set-up of a run (see s2d_setup.h).
//
// The expressions keep the reference's mix of float and double: a float
// quotient rounded before promotion, float overloads of sqrt and exp where
// the reference's argument is a float, and double elsewhere.
#include "s2d_setup.h"

#include <cmath>

namespace s2d {

static const double kPi = 3.141592654;  // cpumodelling.cpp:9

RunSteps derive_steps(const s2d_wave &w, float dx, float dz) {
    RunSteps r;
    const float inv_dx = 1.0f / dx, inv_dz = 1.0f / dz;
    r.fd_nt = (int)std::ceil(w.rec_len / w.fd_dt);      // float quotient, float ceil
    r.real_nt = (int)std::ceil(w.rec_len / w.real_dt);
    r.dtdx = (double)(w.fd_dt * inv_dx);
    r.dtdz = (double)(w.fd_dt * inv_dz);
    r.dt_factor = (int)(w.real_dt / w.fd_dt);
    const double td = std::sqrt(6.0f) / (kPi * w.dom_freq);  // float sqrt, as the reference's sqrt(6.0f)
    r.nts = (int)(5.0f * td / w.fd_dt) + 1;
    if (r.nts > r.fd_nt) r.nts = r.fd_nt;
    return r;
}

std::vector<double> ricker(const s2d_wave &w, int nts) {
    std::vector<double> out(nts > 0 ? nts : 0);
    const double fm = (double)w.dom_freq;
    const double t0 = 1.5 * std::sqrt(6.0) / (kPi * fm);
    for (int i = 0; i < nts; ++i) {
        const double t = (double)(i * w.fd_dt);  // float product first
        const double a = kPi * fm * (t - t0);
        const double a2 = a * a;
        out[i] = (1.0f - 2.0f * a2) * std::exp(-a2);
    }
    return out;
}

static void taper_pair(float t, float &d, float &d1) {
    d = std::exp(-(t * t));                       // float overload
    d1 = (float)std::exp(-0.5 * (double)(t * t)); // double overload
}

void sponge_a(int nb, int n, std::vector<float> &damp, std::vector<float> &damp1) {
    const float fac = 0.05f;  // cpumodelling.cpp:254
    damp.assign(2 * nb + n, 0.0f);
    damp1.assign(2 * nb + n, 0.0f);
    std::vector<float> s(nb), s1(nb);
    for (int i = 0; i < nb; ++i) taper_pair(fac * (float)(nb - (i + 1)), s[i], s1[i]);
    for (int i = 0; i < nb; ++i) {
        damp[i] = s[i];
        damp1[i] = s1[i];
        damp[nb + n + i] = s[nb - i - 1];
        damp1[nb + n + i] = s1[nb - i - 1];
    }
    for (int i = 0; i < n; ++i) damp[nb + i] = damp1[nb + i] = 1.0f;
}

void sponge_b(int nb, int n, std::vector<float> &damp, std::vector<float> &damp1) {
    const float fac = 0.05f;
    damp.assign(2 * nb + n, 0.0f);
    damp1.assign(2 * nb + n, 0.0f);
    for (int i = 0; i < nb - 1; ++i) taper_pair(fac * ((float)(nb - 1 - (i + 1)) + 0.5f), damp[i], damp1[i]);
    for (int i = 0; i < n + 1; ++i) damp[nb - 1 + i] = damp1[nb - 1 + i] = 1.0f;
    for (int i = 0; i < nb; ++i) taper_pair(fac * ((float)i + 0.5f), damp[nb + n + i], damp1[nb + n + i]);
}

void cell_of(float x, float z, float dx, float dz, int nb, int &ix, int &iz) {
    const float inv_dx = 1.0f / dx, inv_dz = 1.0f / dz;
    ix = (int)(x * inv_dx) + nb;
    iz = (int)(z * inv_dz) + nb;
}

}  // namespace s2d

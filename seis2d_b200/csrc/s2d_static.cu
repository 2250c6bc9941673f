// s2d_forward_static: one shot of forward modelling that allocates no device
// memory.
//
// Who needs it.  Some callers cannot call cudaMalloc when they want a shot
// modelled: a service that reserves all of its device memory at start-up and
// forbids allocation afterwards, a program whose own allocator already owns
// the device memory (so a cudaMalloc from this library would fail or fragment
// it), or a latency-critical loop that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree imply.  s2d_forward (which allocates the
// wavefields of each batch, pooled per context) cannot serve them.
//
// How.  Everything the run needs on the device -- wavefields, materials,
// coefficient tables, receiver tables, launch arguments and, for host
// buffers, staging copies of the model and the seismogram -- is carved out of
// one file-scope __device__ array of S2D_STATIC_SCRATCH_BYTES, which every GPU
// that loads the library holds until the process exits.  Jobs that need more
// are rejected with S2D_ERR_NOMEM and a message giving the size they need.
//
// The array is shared by every call on a device and keeps the contents of the
// last call; each call clears what must start at zero.  Calls whose device
// work overlaps on one GPU (from several threads or several streams) race on
// the array and must not be issued.
//
// The array's address: host code cannot use the symbol's name as a device
// address, so the first call on each device looks it up with
// cudaGetSymbolAddress (with that device current) and caches it.  That first
// call may load the library's device code and should come before any stream
// capture is started on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/seis2d.h"
#include "s2d_internal.h"
#include "s2d_setup.h"

namespace s2d {
namespace {

constexpr size_t kScratchBytes = (size_t)S2D_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

int say(char *buf, size_t len, int code, const char *fmt, ...) {
    if (buf && len) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, len, fmt, ap);
        va_end(ap);
    }
    return code;
}

// Device address of g_static_scratch on `device` (which must be current).
int scratch_address(int device, unsigned char **out, char *eb, size_t el) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return say(eb, el, S2D_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s",
                       cudaGetErrorString(e));
        g_scratch_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_ptr[device];
    return S2D_OK;
}

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Carve {
    size_t used = 0;
    template <class T> size_t take(size_t n) {
        const size_t off = used;
        used += (n * sizeof(T) + 255) / 256 * 256;
        return off;
    }
};

}  // namespace
}  // namespace s2d

using namespace s2d;

extern "C" int s2d_forward_static(int device, int nx, int nz, float dx, float dz, int nb, const float *vp,
                                  const float *rho, const s2d_wave *wave, const s2d_shot *shot, float *seis_out,
                                  unsigned flags, void *stream_, char *errbuf, size_t errlen) {
    char *eb = errbuf;
    const size_t el = errlen;
    if (eb && el) eb[0] = 0;
    if (!vp || !rho || !wave || !shot || !seis_out) return say(eb, el, S2D_ERR_ARG, "null argument");
    if (nx < 1 || nz < 1 || nb < 2 || !(dx > 0) || !(dz > 0))
        return say(eb, el, S2D_ERR_ARG, "bad model shape nx=%d nz=%d nb=%d", nx, nz, nb);
    if (!(wave->fd_dt > 0) || !(wave->real_dt > 0) || !(wave->rec_len > 0) || !(wave->dom_freq > 0))
        return say(eb, el, S2D_ERR_ARG, "wave parameters must be positive");
    if (shot->nrec < 0 || (shot->nrec > 0 && !shot->rec)) return say(eb, el, S2D_ERR_ARG, "bad receiver list");
    if (flags & ~(S2D_STATIC_MODEL_DEVICE | S2D_STATIC_SEIS_DEVICE))
        return say(eb, el, S2D_ERR_ARG,
                   "s2d_forward_static: unsupported flag bits 0x%x (accepted: S2D_STATIC_MODEL_DEVICE, "
                   "S2D_STATIC_SEIS_DEVICE; no free surface or 8th-order operator here)",
                   flags & ~(S2D_STATIC_MODEL_DEVICE | S2D_STATIC_SEIS_DEVICE));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return say(eb, el, S2D_ERR_NODEV, "no CUDA device");
    }
    if (device < 0 || device >= ndev || device >= kMaxDevices) return say(eb, el, S2D_ERR_ARG, "bad device %d", device);

    const RunSteps rs = derive_steps(*wave, dx, dz);
    if (rs.fd_nt < 1 || rs.real_nt < 1 || rs.dt_factor < 1) return say(eb, el, S2D_ERR_ARG, "bad time stepping");
    const int nnx = nx + 2 * nb, nnz = nz + 2 * nb;
    const int ld = leading_dim(nnz), nxa = nnx + 2 * S2D_GX;
    const size_t F = (size_t)nxa * ld;
    const int nrec = shot->nrec;
    const bool host_model = !(flags & S2D_STATIC_MODEL_DEVICE), host_seis = !(flags & S2D_STATIC_SEIS_DEVICE);

    // positions (reference float rules) and receiver tables grouped by column
    int sx, sz;
    cell_of(shot->src.x, shot->src.z, dx, dz, nb, sx, sz);
    if (sx < 0 || sx >= nnx || sz < 0 || sz >= nnz)
        return say(eb, el, S2D_ERR_GEOM, "source (%g, %g) m is outside the grid", shot->src.x, shot->src.z);
    std::vector<int> rx(nrec), rz(nrec), ptr(nnx + 1, 0), ez(std::max(nrec, 1)), eid(std::max(nrec, 1));
    for (int g = 0; g < nrec; ++g) {
        cell_of(shot->rec[g].x, shot->rec[g].z, dx, dz, nb, rx[g], rz[g]);
        if (rx[g] < 0 || rx[g] >= nnx || rz[g] < 0 || rz[g] >= nnz)
            return say(eb, el, S2D_ERR_GEOM, "receiver %d (%g, %g) m is outside the grid", g, shot->rec[g].x,
                       shot->rec[g].z);
        ptr[rx[g] + 1]++;
    }
    for (int x = 0; x < nnx; ++x) ptr[x + 1] += ptr[x];
    {
        std::vector<int> fill(ptr.begin(), ptr.end() - 1);
        for (int g = 0; g < nrec; ++g) {
            const int k = fill[rx[g]]++;
            ez[k] = rz[g];
            eid[k] = g;
        }
    }

    // carve the scratch
    Carve cv;
    const size_t o_args = cv.take<StepArgs>(1), o_shot = cv.take<ShotDev>(1), o_group = cv.take<GroupDev>(1);
    const size_t o_err = cv.take<int>(1);
    const size_t o_xc = cv.take<float4>(nxa), o_zc = cv.take<float4>(ld);
    const size_t o_amp = cv.take<float>(rs.fd_nt);
    const size_t o_ptr = cv.take<int>(nnx + 1), o_rz = cv.take<int>(std::max(nrec, 1)),
                 o_rid = cv.take<int>(std::max(nrec, 1));
    const size_t o_vp = host_model ? cv.take<float>((size_t)nx * nz) : 0;
    const size_t o_rho = host_model ? cv.take<float>((size_t)nx * nz) : 0;
    // kappa, bx, bz and the 8 state fields each one block, fields F apart
    // (the kernels address them from one base, ShotDev::fstride)
    const size_t o_kap = cv.take<float>(3 * F), o_bx = o_kap + F * sizeof(float), o_bz = o_kap + 2 * F * sizeof(float);
    const size_t o_bue = cv.take<float>(F);
    size_t o_st[8];
    o_st[0] = cv.take<float>(8 * F);
    for (int f = 1; f < 8; ++f) o_st[f] = o_st[0] + (size_t)f * F * sizeof(float);
    const size_t seis_n = (size_t)nrec * rs.real_nt;
    const size_t o_seis = host_seis ? cv.take<float>(std::max<size_t>(seis_n, 1)) : 0;
    if (cv.used > kScratchBytes)
        return say(eb, el, S2D_ERR_NOMEM,
                   "s2d_forward_static: this job needs %zu bytes of device scratch (padded grid %d x %d, %d receivers "
                   "x %d samples); the static scratch holds %zu bytes",
                   cv.used, nnx, nnz, nrec, rs.real_nt, kScratchBytes);

    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return say(eb, el, S2D_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream_);
    unsigned char *base = nullptr;
    int rc = scratch_address(device, &base, eb, el);
    cudaError_t e = cudaSuccess;
#define SCK(call)                                                                                       \
    do {                                                                                                \
        if (rc == S2D_OK) {                                                                             \
            e = (call);                                                                                 \
            if (e != cudaSuccess) rc = say(eb, el, S2D_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e)); \
        }                                                                                               \
    } while (0)
    auto at = [&](size_t off) { return base + off; };

    // host-side tables (reference-exact set-up)
    std::vector<float> d2a, d2a1, d2b, d2b1, d1a, d1a1, d1b, d1b1;
    sponge_a(nb, nx, d2a, d2a1);
    sponge_b(nb, nx, d2b, d2b1);
    sponge_a(nb, nz, d1a, d1a1);
    sponge_b(nb, nz, d1b, d1b1);
    std::vector<float4> xc(nxa, make_float4(0, 0, 0, 0)), zc(ld, make_float4(0, 0, 0, 0));
    for (int x = 0; x < nnx; ++x)
        xc[x + S2D_GX] = make_float4(d2a[x], (float)(rs.dtdx * d2a1[x]), d2b[x], (float)(rs.dtdx * d2b1[x]));
    for (int z = 0; z < nnz; ++z)
        zc[z + S2D_GZ] = make_float4(d1a[z], (float)(rs.dtdz * d1a1[z]), d1b[z], (float)(rs.dtdz * d1b1[z]));
    const std::vector<double> w = ricker(*wave, rs.nts);
    // kappa = vp^2 rho in double at the source's model cell
    const int mx = std::min(std::max(sx - nb, 0), nx - 1), mz = std::min(std::max(sz - nb, 0), nz - 1);
    float vr[2] = {0, 0};
    if (host_model) {
        vr[0] = vp[(size_t)mx * nz + mz];
        vr[1] = rho[(size_t)mx * nz + mz];
    } else {
        SCK(cudaMemcpy(&vr[0], vp + (size_t)mx * nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
        SCK(cudaMemcpy(&vr[1], rho + (size_t)mx * nz + mz, sizeof(float), cudaMemcpyDeviceToHost));
    }
    const double ksrc = ((double)vr[0] * (double)vr[0]) * (double)vr[1];
    std::vector<float> amp(rs.fd_nt, 0.0f);
    for (int kt = 0; kt < rs.fd_nt && kt <= rs.nts; ++kt)
        amp[kt] = (float)(wave->fd_dt * (kt < rs.nts ? w[kt] : 0.0) * ksrc / (dx * dz));

    // device contents: clear what must start at zero, copy tables and model
    SCK(cudaMemsetAsync(at(o_err), 0, sizeof(int), st));
    SCK(cudaMemsetAsync(at(o_kap), 0, (o_st[0] - o_kap), st));            // materials (and bue) incl. ghosts
    SCK(cudaMemsetAsync(at(o_st[0]), 0, (o_st[7] + F * sizeof(float)) - o_st[0], st));  // 8 state fields
    if (host_seis) SCK(cudaMemsetAsync(at(o_seis), 0, std::max<size_t>(seis_n, 1) * sizeof(float), st));
    else SCK(cudaMemsetAsync(seis_out, 0, seis_n * sizeof(float), st));
    SCK(cudaMemcpyAsync(at(o_xc), xc.data(), sizeof(float4) * nxa, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(at(o_zc), zc.data(), sizeof(float4) * ld, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(at(o_amp), amp.data(), sizeof(float) * rs.fd_nt, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(at(o_ptr), ptr.data(), sizeof(int) * (nnx + 1), cudaMemcpyHostToDevice, st));
    if (nrec) {
        SCK(cudaMemcpyAsync(at(o_rz), ez.data(), sizeof(int) * nrec, cudaMemcpyHostToDevice, st));
        SCK(cudaMemcpyAsync(at(o_rid), eid.data(), sizeof(int) * nrec, cudaMemcpyHostToDevice, st));
    }
    const float *vp_d = vp, *rho_d = rho;
    if (host_model) {
        SCK(cudaMemcpyAsync(at(o_vp), vp, sizeof(float) * nx * nz, cudaMemcpyHostToDevice, st));
        SCK(cudaMemcpyAsync(at(o_rho), rho, sizeof(float) * nx * nz, cudaMemcpyHostToDevice, st));
        vp_d = reinterpret_cast<const float *>(at(o_vp));
        rho_d = reinterpret_cast<const float *>(at(o_rho));
    }
    if (rc == S2D_OK) {
        int k = launch_prepare_model(vp_d, rho_d, nx, nz, nb, ld, reinterpret_cast<float *>(at(o_kap)),
                                     reinterpret_cast<float *>(at(o_bue)), reinterpret_cast<float *>(at(o_bx)),
                                     reinterpret_cast<float *>(at(o_bz)), st);
        if (k) rc = say(eb, el, S2D_ERR_CUDA, "model preparation launch: %s", cudaGetErrorString((cudaError_t)k));
    }

    // one shot, one group; the plain-load step kernel needs no dynamic shared memory
    ShotDev sd;
    std::memset(&sd, 0, sizeof sd);
    for (int par = 0; par < 2; ++par)
        for (int f = 0; f < 4; ++f) sd.st[par][f] = reinterpret_cast<float *>(at(o_st[par * 4 + f]));
    sd.fstride = (int)F;
    sd.kappa = reinterpret_cast<const float *>(at(o_kap));
    sd.bx = reinterpret_cast<const float *>(at(o_bx));
    sd.bz = reinterpret_cast<const float *>(at(o_bz));
    sd.xcoef = reinterpret_cast<const float4 *>(at(o_xc));
    sd.zcoef = reinterpret_cast<const float4 *>(at(o_zc));
    sd.nnx = nnx;
    sd.nnz = nnz;
    sd.ld = ld;
    sd.src_x = sx;
    sd.src_z = sz;
    sd.amp = reinterpret_cast<const float *>(at(o_amp));
    sd.rec_ptr = reinterpret_cast<const int *>(at(o_ptr));
    sd.rec_z = reinterpret_cast<const int *>(at(o_rz));
    sd.rec_id = reinterpret_cast<const int *>(at(o_rid));
    sd.seis = host_seis ? reinterpret_cast<float *>(at(o_seis)) : seis_out;
    sd.real_nt = rs.real_nt;
    sd.nfield = F;          // sizes for the kernels' self-checks (S2D_DEVICE_CHECKS builds)
    sd.nrec = nrec;
    sd.nseis = seis_n;
    sd.zfast_lo = sd.zfast_hi = 0;  // every strip takes the general row path
    sd.xfast_lo = sd.xfast_hi = 0;  // and every column the general column path
    sd.rec_zlo = 0;                 // receivers anywhere
    sd.rec_zhi = nnz - 1;
    int bps = 1;
    if (rc == S2D_OK && (step_kernel_occupancy(kVariantLdg, 128, 0, &bps) || bps < 1)) bps = 1;
    int sms = 1;
    if (rc == S2D_OK) SCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int nstrips = num_strips(nnz);
    const long resident_warps = (long)sms * bps * 4;
    int seg_len = 16;
    for (int L : {512, 256, 128, 64, 32, 16}) {
        if ((long)nstrips * ((nnx + L - 1) / L) >= 4 * resident_warps) {
            seg_len = std::min(L, nnx);
            break;
        }
    }
    GroupDev gd{};
    gd.task_begin = 0;
    gd.nshots = 1;
    gd.shot0 = 0;
    gd.nstrips = nstrips;
    gd.seg_len = seg_len;
    gd.nsegs = (nnx + seg_len - 1) / seg_len;
    SCK(cudaMemcpyAsync(at(o_shot), &sd, sizeof sd, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(at(o_group), &gd, sizeof gd, cudaMemcpyHostToDevice, st));
    StepArgs a{};
    a.shots = reinterpret_cast<const ShotDev *>(at(o_shot));
    a.groups = reinterpret_cast<const GroupDev *>(at(o_group));
    a.ngroups = 1;
    a.total_tasks = gd.nstrips * gd.nsegs;
    a.dt_factor = rs.dt_factor;
    a.fd_nt = rs.fd_nt;
    a.kt_base = 0;
    a.stages = 2;
    a.err = reinterpret_cast<int *>(at(o_err));
    a.spin_limit = 1 << 20;
    a.fault_iter = -1;
    a.task_order = 1;
    StepArgs *args_d = reinterpret_cast<StepArgs *>(at(o_args));
    if (rc == S2D_OK) {
        int k = launch_set_args(a, args_d, st);
        if (k) rc = say(eb, el, S2D_ERR_CUDA, "argument launch: %s", cudaGetErrorString((cudaError_t)k));
    }
    const int grid = (int)std::max<long>(1, std::min<long>((long)sms * bps, ((long)a.total_tasks * 32 + 127) / 128));
    for (int kt = 0; kt < rs.fd_nt && rc == S2D_OK; ++kt) {
        int k = launch_step(kVariantLdg, args_d, kt, grid, 128, 0, st);
        if (k) rc = say(eb, el, S2D_ERR_CUDA, "step launch: %s", cudaGetErrorString((cudaError_t)k));
    }
    if (host_seis && seis_n)
        SCK(cudaMemcpyAsync(seis_out, at(o_seis), seis_n * sizeof(float), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    // the step kernel's device error word: nonzero only when a self-check of a
    // S2D_DEVICE_CHECKS build skipped a task (the plain-load kernel has no waits)
    int dev_err = 0;
    SCK(cudaMemcpy(&dev_err, at(o_err), sizeof(int), cudaMemcpyDeviceToHost));
    if (rc == S2D_OK && dev_err)
        rc = say(eb, el, S2D_ERR_CUDA, "s2d_forward_static: device self-check failed (error word 0x%x)", dev_err);
#undef SCK
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

// Host driver of libseis2d: SeisAcoMod2D's job card, geometry files, model
// files and seismogram files, above the C ABI.
//
// Each routine follows the reference's host code (src/src_cpu/...):
//   job card          json_parser.cpp:13-300
//   shot file         create_geometry.cpp:15-444
//   explicit geometry read_receiver.cpp:14-306
//   model files       model.cpp:12-64
//   stability check   check_stability.cpp:8-72
//   restart, output   cpumodelling.cpp:294-321, 370-374; gpumodelling.cu:471-477
// Where the reference aborts the process (MPI::COMM_WORLD.Abort(code)) these
// return an S2D_ERR_* status and put the reference's abort code in the
// message ("reference code -13").
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/seis2d.h"
#include "s2d_setup.h"

namespace {

int say(char *buf, size_t len, int code, const char *fmt, ...) {
    if (buf && len) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, len, fmt, ap);
        va_end(ap);
    }
    return code;
}

void copy_str(char *dst, size_t cap, const std::string &s) {
    std::snprintf(dst, cap, "%s", s.c_str());
}

// std::stoi / std::stof semantics of the reference (json_parser.cpp:92-120,
// create_geometry.cpp:148-190): leading whitespace skipped, the longest valid
// prefix converted, trailing characters ignored; no conversion is an error.
bool to_int(const std::string &t, int &v) {
    if (t.empty()) return false;
    const char *s = t.c_str();
    char *end = nullptr;
    errno = 0;
    long r = std::strtol(s, &end, 10);
    if (end == s || errno == ERANGE || r > 2147483647L || r < -2147483648L) return false;
    v = (int)r;
    return true;
}
bool to_float(const std::string &t, float &v) {
    if (t.empty()) return false;
    const char *s = t.c_str();
    char *end = nullptr;
    errno = 0;
    float r = std::strtof(s, &end);
    if (end == s || errno == ERANGE) return false;
    v = r;
    return true;
}

// "<dir>/<name>.<ext>" -> "<name>_" (json_parser.cpp:13-37)
std::string job_name(const std::string &path) {
    std::string base = path;
    const size_t slash = base.rfind('/');
    if (slash != std::string::npos) base = base.substr(slash + 1);
    const size_t dot = base.rfind('.');
    if (dot != std::string::npos) base = base.substr(0, dot);
    return base + "_";
}

// remquof remainder truncated to int must be 0 (create_geometry.cpp:192-219)
bool on_grid(float v, float d) {
    int q;
    return (int)remquof(v, d, &q) == 0;
}

}  // namespace

extern "C" {

int s2d_jobcard_read(const char *path, s2d_jobcard *out, char *eb, size_t el) {
    if (!path || !out) return say(eb, el, S2D_ERR_ARG, "null argument");
    std::memset(out, 0, sizeof *out);
    FILE *f = std::fopen(path, "r");
    if (!f) return say(eb, el, S2D_ERR_IO, "unable to open job card %s (reference code -2)", path);
    // json_parser.cpp:40-83: one "key" : "value" per line; comment lines skipped;
    // the first occurrence of a key wins.
    std::map<std::string, std::string> kv;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        if (std::strstr(line, "\"") && std::strstr(line, ":") && !std::strstr(line, "comment") &&
            !std::strstr(line, "Comment")) {
            char key[32] = {0}, val[224] = {0};
            std::sscanf(line, " \"%31[^\"]\" : \"%223[^\"]\" ", key, val);
            kv.insert({key, val});
        }
    }
    std::fclose(f);
    auto need = [&](const char *k, std::string &v) -> bool {
        auto it = kv.find(k);
        if (it == kv.end()) return false;
        v = it->second;
        return true;
    };
    std::string v;
    // json_parser.cpp:122-265
    if (!need("Velocity", v)) return say(eb, el, S2D_ERR_JOBCARD, "missing velocity file name (reference code -6)");
    copy_str(out->velfile, sizeof out->velfile, v);
    if (!need("Density", v)) return say(eb, el, S2D_ERR_JOBCARD, "missing density file name (reference code -6)");
    copy_str(out->densfile, sizeof out->densfile, v);
    if (!need("NX", v) || !to_int(v, out->nx))
        return say(eb, el, S2D_ERR_JOBCARD, "missing NX (number of grid points in X direction) (reference code -6)");
    if (!need("NZ", v) || !to_int(v, out->nz))
        return say(eb, el, S2D_ERR_JOBCARD, "missing NZ (number of grid points in Z direction) (reference code -6)");
    if (!need("DX", v) || !to_float(v, out->dx))
        return say(eb, el, S2D_ERR_JOBCARD, "missing grid spacing in X direction (reference code -6)");
    if (!need("DZ", v) || !to_float(v, out->dz))
        return say(eb, el, S2D_ERR_JOBCARD, "missing grid spacing in Z direction (reference code -6)");
    if (!need("Time", v) || !to_float(v, out->wave.rec_len))
        return say(eb, el, S2D_ERR_JOBCARD, "missing record time (reference code -6)");
    if (!need("FD DT", v) || !to_float(v, out->wave.fd_dt))
        return say(eb, el, S2D_ERR_JOBCARD, "missing FD sampling interval (DT) (reference code -6)");
    if (!need("DATA DT", v) || !to_float(v, out->wave.real_dt))
        return say(eb, el, S2D_ERR_JOBCARD, "missing seismogram sampling interval (DT) (reference code -6)");
    if (std::fmod(out->wave.real_dt, out->wave.fd_dt) != 0)
        return say(eb, el, S2D_ERR_JOBCARD,
                   "DATA DT must be multiple of FD DT (DATA_DT>=FD_DT & DATA_DT%%FD_DT=0) (reference code -6)");
    if (!need("Frequency", v) || !to_float(v, out->wave.dom_freq))
        return say(eb, el, S2D_ERR_JOBCARD, "missing dominant frequency (reference code -6)");
    if (!need("Read source receiver flag", v) || !to_int(v, out->geomflag))
        return say(eb, el, S2D_ERR_JOBCARD, "missing read source-receiver flag (reference code -6)");
    if (out->geomflag < 0 || out->geomflag > 1)
        return say(eb, el, S2D_ERR_JOBCARD, "wrong flag value for read source-receiver flag (reference code -6)");
    if (out->geomflag == 0) {
        if (!need("if choice=0, Geometry file", v))
            return say(eb, el, S2D_ERR_JOBCARD, "missing source-receiver geometry file name (reference code -6)");
        copy_str(out->geomfile, sizeof out->geomfile, v);
    } else {
        if (!need("if choice=1, Shot file", v))
            return say(eb, el, S2D_ERR_JOBCARD, "missing shot file name (reference code -6)");
        copy_str(out->shotfile, sizeof out->shotfile, v);
    }
    if (!need("Output Directory", v))
        return say(eb, el, S2D_ERR_JOBCARD, "missing Output directory path (reference code -6)");
    if (v.empty() || v.back() != '/') v += "/";
    copy_str(out->tmppath, sizeof out->tmppath, v);
    if (!need("Free surface", v) || !to_int(v, out->frsf))
        return say(eb, el, S2D_ERR_JOBCARD, "missing free surface flag (reference code -6)");
    if (out->frsf < 0 || out->frsf > 1)
        return say(eb, el, S2D_ERR_JOBCARD, "wrong flag value for free surface choice (reference code -6)");
    if (!need("Job type New or Restart", v))
        return say(eb, el, S2D_ERR_JOBCARD, "missing job type New or Restart (reference code -6)");
    if (v != "New" && v != "Restart")
        return say(eb, el, S2D_ERR_JOBCARD, "wrong value is specified for job status (reference code -6)");
    copy_str(out->jbtype, sizeof out->jbtype, v);
    if (!need("Order of FD Operator", v) || !to_int(v, out->fdop))
        return say(eb, el, S2D_ERR_JOBCARD, "missing order of FD Operator (reference code -6)");
    copy_str(out->jobname, sizeof out->jobname, job_name(path));
    return S2D_OK;
}

void s2d_geometry_free(s2d_geometry *g) {
    if (!g) return;
    if (g->rec)
        for (int s = 0; s < g->nsrc; ++s) std::free(g->rec[s]);
    std::free(g->rec);
    std::free(g->nrec);
    std::free(g->src);
    std::memset(g, 0, sizeof *g);
}

}  // extern "C"

namespace {

// Receivers of one shot from a shot-file line (create_geometry.cpp:237-444).
// The reference steps the receiver position in float (i += spacing) and
// writes into an array of nrec zero-initialised entries; positions the loop
// skips stay (0, 0), and positions past the nrec-th are not kept (the
// reference writes them past the end of its array).
int make_receivers(const s2d_jobcard &J, float sx, float sz, int nrec, float nearoff, float d, int type,
                   s2d_coord *rec, char *eb, size_t el) {
    const float xmax = (J.nx - 1) * J.dx;
    // check_geom_para (create_geometry.cpp:192-235)
    if (!on_grid(sx, J.dx))
        return say(eb, el, S2D_ERR_GEOM, "source x %g is not a multiple of dx (reference code -13)", sx);
    if (!on_grid(sz, J.dz))
        return say(eb, el, S2D_ERR_GEOM, "source z %g is not a multiple of dz (reference code -14)", sz);
    if (!on_grid(d, J.dx))
        return say(eb, el, S2D_ERR_GEOM, "receiver spacing %g is not a multiple of dx (reference code -15)", d);
    if (sx < 0 || sx > xmax) return say(eb, el, S2D_ERR_GEOM, "source x %g outside the model (reference code -16)", sx);
    if (sz < 0 || sz > (J.nz - 1) * J.dz)
        return say(eb, el, S2D_ERR_GEOM, "source z %g outside the model (reference code -17)", sz);
    float start, end;
    if (type == 1) {  // split (create_geometry.cpp:265-355)
        const int tmp1 = (int)((sx - 0.0f) / d);
        const int tmp2 = (int)((xmax - sx) / d);
        if (nearoff == 0.0f) {
            if (tmp1 < nrec / 2) {
                start = sx - (tmp1 * d);
                end = start + ((nrec - 1) * d);
            } else if (tmp2 < nrec / 2) {
                start = sx - ((nrec - tmp2 - 1) * d);
                end = start + ((nrec - 1) * d);
            } else {
                start = sx - ((nrec / 2) * d);
                end = start + ((nrec - 1) * d);
            }
        } else {
            if (tmp1 < nrec / 2) {
                start = sx - (tmp1 * d);
                end = start + ((nrec - 1) * d) + d;
            } else if (tmp2 < nrec / 2) {
                start = sx - ((nrec - tmp2) * d);
                end = start + (nrec * d);
            } else {
                start = sx - ((nrec / 2) * d);
                end = start + ((nrec - 1) * d);
                if ((start - d) >= 0) start -= d;
                else end += d;
            }
        }
    } else if (type == 2) {  // end-on left (create_geometry.cpp:357-399)
        end = nearoff == 0.0f ? sx : sx - d;
        start = end - ((nrec - 1) * d);
    } else if (type == 3) {  // end-on right (create_geometry.cpp:401-444)
        start = nearoff == 0.0f ? sx : sx + d;
        end = start + ((nrec - 1) * d);
    } else {
        return say(eb, el, S2D_ERR_GEOM, "wrong geometry type %d (1 split, 2 end-on-left, 3 end-on-right) "
                   "(reference code -12)", type);
    }
    if (start < 0.0f)
        return say(eb, el, S2D_ERR_GEOM, "receiver x %g goes out of model for source %g,%g (reference code -3)",
                   start, sx, sz);
    if (end > xmax)
        return say(eb, el, S2D_ERR_GEOM, "receiver x %g goes out of model for source %g,%g (reference code -3)", end,
                   sx, sz);
    float i = start;
    int j = 0;
    while (i <= end) {
        const bool write = (type != 1 || nearoff == 0.0f || i != sx);
        if (write && j < nrec) {
            rec[j].x = i;
            rec[j].z = sz;
        }
        i += d;
        j++;
    }
    return S2D_OK;
}

int read_shotfile(const s2d_jobcard &J, s2d_geometry *G, char *eb, size_t el) {
    const char *path = J.shotfile;
    // count shots: lines without "comment" that hold a token (create_geometry.cpp:34-39)
    FILE *f = std::fopen(path, "r");
    if (!f) return say(eb, el, S2D_ERR_IO, "unable to open shot file %s (reference code -2)", path);
    char buf[256], tok[256];
    int nsrc = 0;
    while (std::fgets(buf, sizeof buf, f))
        if (!std::strstr(buf, "comment") && std::sscanf(buf, "%255s", tok) == 1) nsrc++;
    std::fclose(f);
    std::ifstream in(path);
    if (!in.is_open()) return say(eb, el, S2D_ERR_IO, "unable to open shot file %s (reference code -23)", path);
    if (in.peek() == std::ifstream::traits_type::eof())
        return say(eb, el, S2D_ERR_GEOM, "shot file %s is empty (reference code -24)", path);
    G->nsrc = nsrc;
    G->nrec = (int *)std::calloc(std::max(nsrc, 1), sizeof(int));
    G->src = (s2d_coord *)std::calloc(std::max(nsrc, 1), sizeof(s2d_coord));
    G->rec = (s2d_coord **)std::calloc(std::max(nsrc, 1), sizeof(s2d_coord *));
    int default_type = 0;
    for (int s = 0; s < nsrc; ++s) {
        std::string line;
        std::getline(in, line);
        if (line.empty())
            return say(eb, el, S2D_ERR_GEOM, "blank line in shot file %s (reference code -20)", path);
        std::istringstream stm(line);
        std::string t[7];
        int n = 0;
        while (n < 7 && std::getline(stm, t[n], ',')) n++;
        if (n != 6)
            return say(eb, el, S2D_ERR_GEOM, "wrong number of arguments for source number %d: expected "
                       "sx,sz,nrec,nearoff,spacing,type (reference code -25)", s + 1);
        float sx, sz, nearoff, d;
        int nrec, type;
        if (!to_float(t[0], sx) || !to_float(t[1], sz) || !to_int(t[2], nrec) || !to_float(t[3], nearoff) ||
            !to_float(t[4], d) || !to_int(t[5], type))
            return say(eb, el, S2D_ERR_GEOM, "missing information in shot file for source number %d "
                       "(reference code -19)", s + 1);
        if (s == 0) default_type = type;
        if (type != default_type)
            return say(eb, el, S2D_ERR_GEOM, "geophone geometry type must be the same for all shots "
                       "(reference code -11)");
        if (nrec <= 0)
            return say(eb, el, S2D_ERR_GEOM, "number of receivers cannot be zero or negative (reference code -18)");
        G->src[s].x = sx;
        G->src[s].z = sz;
        G->nrec[s] = nrec;
        G->rec[s] = (s2d_coord *)std::calloc(nrec, sizeof(s2d_coord));
        int e = make_receivers(J, sx, sz, nrec, nearoff, d, type, G->rec[s], eb, el);
        if (e) return e;
    }
    return S2D_OK;
}

int check_coord(const s2d_jobcard &J, float sx, float sz, float gx, float gz, char *eb, size_t el) {
    // read_receiver.cpp:93-159
    if (!on_grid(sx, J.dx)) return say(eb, el, S2D_ERR_GEOM, "source x %g not on the grid (reference code -13)", sx);
    if (!on_grid(sz, J.dz)) return say(eb, el, S2D_ERR_GEOM, "source z %g not on the grid (reference code -14)", sz);
    if (!on_grid(gx, J.dx)) return say(eb, el, S2D_ERR_GEOM, "receiver x %g not on the grid (reference code -13)", gx);
    if (!on_grid(gz, J.dz)) return say(eb, el, S2D_ERR_GEOM, "receiver z %g not on the grid (reference code -14)", gz);
    const float xmax = (J.nx - 1) * J.dx, zmax = (J.nz - 1) * J.dz;
    if (sx < 0 || sx > xmax) return say(eb, el, S2D_ERR_GEOM, "source x %g outside the model (reference code -16)", sx);
    if (sz < 0 || sz > zmax) return say(eb, el, S2D_ERR_GEOM, "source z %g outside the model (reference code -17)", sz);
    if (gx < 0 || gx > xmax)
        return say(eb, el, S2D_ERR_GEOM, "receiver x %g outside the model (reference code -16)", gx);
    if (gz < 0 || gz > zmax)
        return say(eb, el, S2D_ERR_GEOM, "receiver z %g outside the model (reference code -17)", gz);
    return S2D_OK;
}

int read_geomfile(const s2d_jobcard &J, s2d_geometry *G, char *eb, size_t el) {
    const char *path = J.geomfile;
    std::ifstream in(path);
    if (!in.is_open()) return say(eb, el, S2D_ERR_IO, "unable to open receiver geometry file %s (reference code -3)", path);
    if (in.peek() == std::ifstream::traits_type::eof())
        return say(eb, el, S2D_ERR_GEOM, "receiver geometry file %s is empty (reference code -4)", path);
    // count_src (read_receiver.cpp:162-306): consecutive lines with the same
    // (sx, sz) form one shot; sx must increase between shots.
    struct Row { float sx, sz, gx, gz; };
    std::vector<Row> rows;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty()) return say(eb, el, S2D_ERR_GEOM, "blank line in receiver geometry file (reference code -21)");
        std::istringstream stm(line);
        std::string t[5];
        int n = 0;
        while (n < 5 && std::getline(stm, t[n], ',')) n++;
        if (n != 4)
            return say(eb, el, S2D_ERR_GEOM, "wrong number of arguments: expected sx,sz,gx,gz (reference code -26)");
        Row r;
        if (!to_float(t[0], r.sx) || !to_float(t[1], r.sz) || !to_float(t[2], r.gx) || !to_float(t[3], r.gz))
            return say(eb, el, S2D_ERR_GEOM, "missing coordinate in receiver geometry file (reference code -19)");
        rows.push_back(r);
    }
    std::vector<int> counts;
    size_t first = 0;  // first row of the current shot: (sx_old, sz_old)
    for (size_t i = 0; i < rows.size(); ++i) {
        if (i == 0) {
            counts.push_back(1);
            continue;
        }
        const Row &b = rows[i], &o = rows[first];
        if (b.sx == o.sx && b.sz == o.sz) {
            counts.back()++;
        } else if (b.sx > o.sx) {
            counts.push_back(1);
            first = i;
        } else {
            return say(eb, el, S2D_ERR_GEOM, "geometry file must be sorted on sx (source x %g after %g) "
                       "(reference code -22)", b.sx, o.sx);
        }
    }
    G->nsrc = (int)counts.size();
    G->nrec = (int *)std::calloc(std::max(G->nsrc, 1), sizeof(int));
    G->src = (s2d_coord *)std::calloc(std::max(G->nsrc, 1), sizeof(s2d_coord));
    G->rec = (s2d_coord **)std::calloc(std::max(G->nsrc, 1), sizeof(s2d_coord *));
    size_t k = 0;
    for (int s = 0; s < G->nsrc; ++s) {
        G->nrec[s] = counts[s];
        G->src[s].x = rows[k].sx;
        G->src[s].z = rows[k].sz;
        G->rec[s] = (s2d_coord *)std::calloc(counts[s], sizeof(s2d_coord));
        for (int g = 0; g < counts[s]; ++g, ++k) {
            // read_receiver.cpp:62-86: the shot's source is taken from its first row
            int e = check_coord(J, G->src[s].x, G->src[s].z, rows[k].gx, rows[k].gz, eb, el);
            if (e) return e;
            G->rec[s][g].x = rows[k].gx;
            G->rec[s][g].z = rows[k].gz;
        }
    }
    return S2D_OK;
}

// model.cpp:12-44: raw float32 [nx][nz]; size check in float arithmetic.
int read_model(const char *path, int nx, int nz, std::vector<float> &out, char *eb, size_t el) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return say(eb, el, S2D_ERR_IO, "unable to open input model %s (reference code -2)", path);
    std::fseek(f, 0, SEEK_END);
    const float file_size = (float)std::ftell(f);
    std::rewind(f);
    const float rem = file_size / (float)(nx * nz);
    if (rem != 4.0f) {
        std::fclose(f);
        return say(eb, el, S2D_ERR_IO, "input file %s is empty or does not hold NX*NZ floats (reference code -2)", path);
    }
    out.resize((size_t)nx * nz);
    const size_t got = std::fread(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
    if (got != out.size()) return say(eb, el, S2D_ERR_IO, "short read of %s", path);
    return S2D_OK;
}

}  // namespace

extern "C" {

int s2d_geometry_read(const s2d_jobcard *job, s2d_geometry *out, char *eb, size_t el) {
    if (!job || !out) return say(eb, el, S2D_ERR_ARG, "null argument");
    std::memset(out, 0, sizeof *out);
    int e = job->geomflag == 0 ? read_geomfile(*job, out, eb, el) : read_shotfile(*job, out, eb, el);
    if (e) s2d_geometry_free(out);
    return e;
}

int s2d_check_stability(const s2d_jobcard *J, float vmin, float vmax, char *eb, size_t el) {
    if (!J) return say(eb, el, S2D_ERR_ARG, "null argument");
    // check_stability.cpp:8-72
    const float fm = 2.0f * J->wave.dom_freq;
    const float hmin = std::min(J->dx, J->dz), hmax = std::max(J->dx, J->dz);
    // 0.606 = 1 / (sqrt(2) (a0 + |a1|)) of the 4th-order operator; the 8th-order
    // operator's coefficient sum 1.2863 gives 0.549 (no counterpart in the reference)
    float criteria = ((J->fdop == 8 ? 0.549f : 0.606f) * hmin) / vmax;
    if (J->wave.fd_dt > criteria)
        return say(eb, el, S2D_ERR_STABILITY, "stability condition violated: dt %g > %g (reference code -5)",
                   J->wave.fd_dt, criteria);
    criteria = vmin / (hmax * 5.0f);
    if (fm > criteria)
        return say(eb, el, S2D_ERR_STABILITY, "non-dispersion relation not satisfied: peak frequency %g > %g "
                   "(reference code -5)", J->wave.dom_freq, criteria / 2.0f);
    return S2D_OK;
}

int s2d_workload(int nsrc, int nranks, int rank, int *start, int *count) {
    if (!start || !count || nranks < 1 || rank < 0 || rank >= nranks || nsrc < 0) return S2D_ERR_ARG;
    // workload.cpp:21-31: fewer sources than ranks is an error (abort -8 there)
    if (nsrc < nranks) return S2D_ERR_ARG;
    // workload.cpp:34-48: contiguous blocks, the first nsrc % nranks one longer
    const int div = nsrc / nranks, mod = nsrc % nranks;
    *start = rank * div + std::min(rank, mod);
    *count = div + (rank < mod ? 1 : 0);
    return S2D_OK;
}

int s2d_run_jobcard(const char *jobcard_path, int device, int nb, int naming, int check_stability, int verbose,
                    char *eb, size_t el) {
    return s2d_run_jobcard_rank(jobcard_path, device, nb, naming, check_stability, verbose, 0, 1, eb, el);
}

int s2d_run_jobcard_rank(const char *jobcard_path, int device, int nb, int naming, int check_stability, int verbose,
                         int rank, int nranks, char *eb, size_t el) {
    s2d_jobcard J;
    int e = s2d_jobcard_read(jobcard_path, &J, eb, el);
    if (e) return e;
    // 4: the reference's operator; 8: the 8th-order operator (the reference
    // parses the key and steps only for 4, cpumodelling.cpp:121)
    if (J.fdop != 4 && J.fdop != 8)
        return say(eb, el, S2D_ERR_JOBCARD, "FD operators of order 4 and 8 exist (Order of FD Operator = %d)",
                   J.fdop);
    s2d_geometry G;
    e = s2d_geometry_read(&J, &G, eb, el);
    if (e) return e;
    std::vector<float> vp, rho;
    e = read_model(J.velfile, J.nx, J.nz, vp, eb, el);
    if (!e) e = read_model(J.densfile, J.nx, J.nz, rho, eb, el);
    if (e) {
        s2d_geometry_free(&G);
        return e;
    }
    // minmax2d (model.cpp:47-64)
    float vmin = vp[0], vmax = vp[0];
    for (float v : vp) {
        if (v < vmin) vmin = v;
        if (v > vmax) vmax = v;
    }
    if (check_stability) {
        e = s2d_check_stability(&J, vmin, vmax, eb, el);
        if (e) {
            s2d_geometry_free(&G);
            return e;
        }
    }
    // this rank's block of shots (workload.cpp:12-62)
    int first = 0, nmine = 0;
    if (s2d_workload(G.nsrc, nranks, rank, &first, &nmine) != S2D_OK) {
        s2d_geometry_free(&G);
        if (nranks >= 1 && rank >= 0 && rank < nranks && G.nsrc < nranks)
            return say(eb, el, S2D_ERR_ARG,
                       "number of sources (%d) should be greater than or equal to the number of ranks (%d) "
                       "(reference code -8)", G.nsrc, nranks);
        return say(eb, el, S2D_ERR_ARG, "bad rank %d of %d", rank, nranks);
    }
    // restart index (cpumodelling.cpp:294-321): per rank, an index into the
    // rank's own shots; this driver also writes it after every completed
    // shot, which the reference never does
    const std::string ckpt = std::string(J.tmppath) + J.jobname + "checkpoint_rank" + std::to_string(rank) + ".txt";
    int istart = 0;
    if (std::strcmp(J.jbtype, "Restart") == 0) {
        FILE *f = std::fopen(ckpt.c_str(), "r");
        if (!f) {
            s2d_geometry_free(&G);
            return say(eb, el, S2D_ERR_IO, "error in opening restart file %s (reference code -10)", ckpt.c_str());
        }
        if (std::fscanf(f, "%d", &istart) != 1) istart = 0;
        std::fclose(f);
        istart = std::max(0, std::min(istart, nmine));
    }
    void *ctx = nullptr;
    e = s2d_create(&ctx, device);
    if (e) {
        s2d_geometry_free(&G);
        return say(eb, el, e, "no usable CUDA device %d", device);
    }
    int mid = 0;
    // "Free surface" : "1" (parsed and ignored by the reference) turns the
    // first model row into a pressure-release surface
    e = s2d_model_create(ctx, J.nx, J.nz, J.dx, J.dz, nb, vp.data(), rho.data(),
                         (J.frsf ? S2D_MODEL_FREE_SURFACE : 0u) | (J.fdop == 8 ? S2D_MODEL_ORDER8 : 0u), &mid);
    s2d_steps st;
    if (!e) e = s2d_derive_steps(&J.wave, &st);
    // shots per batch: what fits in free device memory (8 wavefield buffers per shot)
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const int nnx = J.nx + 2 * nb, nnz = J.nz + 2 * nb;
    const double per_shot = 8.0 * (nnx + 16.0) * (nnz + 136.0) * 4.0 * 1.05;
    int batch = (int)std::max(1.0, std::floor(0.85 * (double)free_b / per_shot));
    for (int s0 = istart; !e && s0 < nmine; s0 += batch) {
        const int n = std::min(batch, nmine - s0);
        std::vector<s2d_shot> shots(n);
        size_t total = 0;
        for (int k = 0; k < n; ++k) {
            const int g = first + s0 + k;
            shots[k].model_id = mid;
            shots[k].src = G.src[g];
            shots[k].nrec = G.nrec[g];
            shots[k].rec = G.rec[g];
            total += (size_t)G.nrec[g] * st.real_nt;
        }
        std::vector<float> seis(total);
        e = s2d_forward(ctx, shots.data(), n, &J.wave, nullptr, 0, 0, 0, seis.data(), 0, nullptr);
        if (e) {
            say(eb, el, e, "%s", s2d_last_error(ctx));
            break;
        }
        size_t off = 0;
        for (int k = 0; k < n && !e; ++k) {
            const int s = first + s0 + k;  // index in the whole geometry
            std::string name = std::string(J.tmppath) + J.jobname;
            if (naming == 1) {
                // gpumodelling.cu:471-477: "sx%.2f" of the source's grid x in metres
                char sxs[64];
                const int ix = (int)(G.src[s].x * (1.0f / J.dx));
                std::snprintf(sxs, sizeof sxs, "sx%.2f", (double)(ix * J.dx));
                name += sxs;
                name += "_";
            }
            name += "seismogram.bin";
            FILE *f = std::fopen(name.c_str(), "wb");
            if (!f) {
                e = say(eb, el, S2D_ERR_IO, "unable to write %s", name.c_str());
                break;
            }
            const size_t cnt = (size_t)G.nrec[s] * st.real_nt;
            std::fwrite(seis.data() + off, sizeof(float), cnt, f);
            std::fclose(f);
            off += cnt;
            FILE *c = std::fopen(ckpt.c_str(), "w");
            if (c) {
                std::fprintf(c, "%d\n", s0 + k + 1);
                std::fclose(c);
            }
            if (verbose) std::printf(" Rank: %d   Shot remaining: %d\n", rank, nmine - (s0 + k + 1));
        }
    }
    s2d_destroy(ctx);
    s2d_geometry_free(&G);
    return e;
}

}  // extern "C"

// Host utilities of the C ABI (no GPU): the reference's binary file formats,
// the synthetic initial state, the reference's created obstacles and the
// host voxeliser (node tests shared with the device, geometry.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/eup.h"
#include "geometry.h"
#include "init_eq.h"

using eup::splitmix64;

// Shared with the device entry points: eup_last_error(NULL) reports it.
void eup_internal_set_error(const std::string& msg);

namespace {

int herr(int code, const std::string& m) {
    eup_internal_set_error(m);
    return code;
}

// ---- Fortran unformatted sequential records (gfortran layout): each record is
// [int32 length][payload][int32 length].  Records above 2^31-9 bytes would be
// split into sub-records; they are rejected here.
struct FFile {
    FILE* f = nullptr;
    explicit FFile(const char* path, const char* mode) { f = std::fopen(path, mode); }
    ~FFile() { if (f) std::fclose(f); }
};

bool read_record(FILE* f, void* dst, int64_t want, std::string& why) {
    int32_t head = 0, tail = 0;
    if (std::fread(&head, 4, 1, f) != 1) { why = "missing record header"; return false; }
    if (head < 0) { why = "Fortran sub-records (records over 2 GiB) are not supported"; return false; }
    if ((int64_t)head != want) {
        why = "record of " + std::to_string(head) + " bytes, expected " + std::to_string(want);
        return false;
    }
    if (want > 0 && std::fread(dst, 1, (size_t)want, f) != (size_t)want) { why = "short record"; return false; }
    if (std::fread(&tail, 4, 1, f) != 1 || tail != head) { why = "bad record trailer"; return false; }
    return true;
}

bool write_record(FILE* f, const void* src, int64_t bytes) {
    if (bytes > 2147483639LL) return false;
    const int32_t m = (int32_t)bytes;
    return std::fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || std::fwrite(src, 1, (size_t)bytes, f) == (size_t)bytes) &&
           std::fwrite(&m, 4, 1, f) == 1;
}


template <typename T>
void init_state(int32_t l, int32_t m, int32_t n, double u_in, double amp, uint64_t seed, void* const pops[19]) {
    const int64_t total = (int64_t)(l + 2) * (m + 2) * (n + 2);
    T* dst[19];
    for (int q = 0; q < 19; ++q) dst[q] = static_cast<T*>(pops[q]);
#pragma omp parallel for schedule(static)
    for (int64_t L = 0; L < total; ++L) {
        T f[19];
        eup::init_node<T>(L, u_in, amp, seed, f);
        for (int q = 0; q < 19; ++q) dst[q][L] = f[q];
    }
}

}  // namespace

// Fortran sequential-record helpers for the device-side checkpoint entry points.
bool eup_internal_read_record(FILE* f, void* dst, int64_t want, std::string* why) {
    return read_record(f, dst, want, *why);
}
bool eup_internal_write_record(FILE* f, const void* src, int64_t bytes) { return write_record(f, src, bytes); }

extern "C" {

int eup_read_obs_file(const char* path, int32_t l, int32_t m, int32_t n, int32_t* obs, int64_t* nobs) {
    if (!path || !obs || l < 1 || m < 1 || n < 1) return herr(EUP_ERR_INVALID_ARG, "eup_read_obs_file: bad argument");
    FFile f(path, "rb");
    if (!f.f) return herr(EUP_ERR_IO, std::string("eup_read_obs_file: cannot open ") + path);
    std::memset(obs, 0, sizeof(int32_t) * (size_t)l * m * n);
    int32_t cnt = 0;
    std::string why;
    if (!read_record(f.f, &cnt, 4, why)) return herr(EUP_ERR_IO, "eup_read_obs_file: header: " + why);
    if (cnt < 0) return herr(EUP_ERR_IO, "eup_read_obs_file: negative obstacle count");
    for (int32_t t = 0; t < cnt; ++t) {
        int32_t ijk[3];
        if (!read_record(f.f, ijk, 12, why)) return herr(EUP_ERR_IO, "eup_read_obs_file: entry " + std::to_string(t) + ": " + why);
        if (ijk[0] < 1 || ijk[0] > l || ijk[1] < 1 || ijk[1] > m || ijk[2] < 1 || ijk[2] > n)
            return herr(EUP_ERR_IO, "eup_read_obs_file: obstacle index out of range");
        obs[(int64_t)(ijk[0] - 1) + (int64_t)l * ((ijk[1] - 1) + (int64_t)m * (ijk[2] - 1))] = 1;
    }
    if (nobs) *nobs = cnt;
    return EUP_OK;
}

int eup_write_obs_file(const char* path, int32_t l, int32_t m, int32_t n, const int32_t* obs) {
    if (!path || !obs || l < 1 || m < 1 || n < 1) return herr(EUP_ERR_INVALID_ARG, "eup_write_obs_file: bad argument");
    const int64_t N = (int64_t)l * m * n;
    int64_t cnt = 0;
    for (int64_t t = 0; t < N; ++t) cnt += (obs[t] == 1);
    if (cnt > 2147483647LL) return herr(EUP_ERR_UNSUPPORTED, "eup_write_obs_file: too many obstacles");
    FFile f(path, "wb");
    if (!f.f) return herr(EUP_ERR_IO, std::string("eup_write_obs_file: cannot open ") + path);
    const int32_t c32 = (int32_t)cnt;
    if (!write_record(f.f, &c32, 4)) return herr(EUP_ERR_IO, "eup_write_obs_file: write failed");
    for (int32_t k = 1; k <= n; ++k)
        for (int32_t j = 1; j <= m; ++j)
            for (int32_t i = 1; i <= l; ++i)
                if (obs[(int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1))] == 1) {
                    const int32_t ijk[3] = {i, j, k};
                    if (!write_record(f.f, ijk, 12)) return herr(EUP_ERR_IO, "eup_write_obs_file: write failed");
                }
    return EUP_OK;
}

int eup_read_raw_state(const char* path, int32_t l, int32_t m, int32_t n, int32_t elem_bytes, void* const pops[19],
                       int64_t* itime) {
    if (!path || !pops || (elem_bytes != 4 && elem_bytes != 8) || l < 1 || m < 1 || n < 1)
        return herr(EUP_ERR_INVALID_ARG, "eup_read_raw_state: bad argument");
    FFile f(path, "rb");
    if (!f.f) return herr(EUP_ERR_IO, std::string("eup_read_raw_state: cannot open ") + path);
    std::string why;
    int32_t it = 0;
    if (!read_record(f.f, &it, 4, why)) return herr(EUP_ERR_IO, "eup_read_raw_state: itime: " + why);
    const int64_t bytes = (int64_t)(l + 2) * (m + 2) * (n + 2) * elem_bytes;
    for (int q = 0; q < 19; ++q) {
        if (!pops[q]) return herr(EUP_ERR_INVALID_ARG, "eup_read_raw_state: null population array");
        if (!read_record(f.f, pops[q], bytes, why))
            return herr(EUP_ERR_IO, "eup_read_raw_state: population " + std::to_string(q + 1) + ": " + why);
    }
    if (itime) *itime = it;
    return EUP_OK;
}

int eup_write_raw_state(const char* path, int32_t l, int32_t m, int32_t n, int32_t elem_bytes,
                        const void* const pops[19], int64_t itime) {
    if (!path || !pops || (elem_bytes != 4 && elem_bytes != 8) || l < 1 || m < 1 || n < 1)
        return herr(EUP_ERR_INVALID_ARG, "eup_write_raw_state: bad argument");
    if (itime < INT32_MIN || itime > INT32_MAX) return herr(EUP_ERR_INVALID_ARG, "eup_write_raw_state: itime overflows int32");
    FFile f(path, "wb");
    if (!f.f) return herr(EUP_ERR_IO, std::string("eup_write_raw_state: cannot open ") + path);
    const int32_t it = (int32_t)itime;
    if (!write_record(f.f, &it, 4)) return herr(EUP_ERR_IO, "eup_write_raw_state: write failed");
    const int64_t bytes = (int64_t)(l + 2) * (m + 2) * (n + 2) * elem_bytes;
    for (int q = 0; q < 19; ++q) {
        if (!pops[q]) return herr(EUP_ERR_INVALID_ARG, "eup_write_raw_state: null population array");
        if (!write_record(f.f, pops[q], bytes))
            return herr(EUP_ERR_IO, "eup_write_raw_state: write failed (records over 2 GiB are not supported)");
    }
    return EUP_OK;
}

}  // extern "C"

namespace {

// One coordinate of CODE/SRC/init.F90:110-133 for index c (0 .. size+1) of a block
// starting at `start` in a lattice of `size` nodes, scaled by `scale` (x is scaled by lz in
// the reference).  Default build: evaluated in default REAL (single precision) whatever
// mykind is; -DPERIODIC: (c + start - 1/2)/size formed in quad precision and rounded to
// mykind, which is one correctly rounded division of exact operands in T.
template <typename T>
T init_coord(int c, int start, int size, int scale, bool periodic) {
    if (periodic) return (T)((T)(c + start) - (T)0.5) / (T)size;
    const float a = (float)(c + start) - 0.5f - 0.5f * (float)size;
    return (T)(a / (0.5f * (float)scale));
}

template <typename T>
void init_reference_t(int opt, int32_t l, int32_t m, int32_t n, const int32_t glob[3], const int32_t start[3],
                      bool periodic, double u0, void* const pops[19]) {
    const T pi = (T)3.141592653589793238462643383279f;  // a default-REAL parameter (:61)
    const T tenth = (T)0.1f, two = (T)2, u0t = (T)u0;
    const int64_t L2 = l + 2, M2 = m + 2;
    T* dst[19];
    for (int q = 0; q < 19; ++q) dst[q] = static_cast<T*>(pops[q]);
#pragma omp parallel for schedule(static)
    for (int32_t k = 0; k <= n + 1; ++k) {
        const T z = init_coord<T>(k, start[2], glob[2], glob[2], periodic);
        for (int32_t j = 0; j <= m + 1; ++j)
            for (int32_t i = 0; i <= l + 1; ++i) {
                const T x = init_coord<T>(i, start[0], glob[0], periodic ? glob[0] : glob[2], periodic);
                T xj = 0, yj = 0, zj = 0;
                if (opt == 1) {
                    xj = tenth * ((T)1 - z * z);  // Poiseuille (:148-152)
                } else if (opt == 2) {
                    xj = u0t * std::sin(two * pi * z);  // decaying flow (:154-161)
                } else if (opt == 3) {            // Kida vortices (:163-171)
                    xj = tenth * std::sin(two * pi * x) * std::cos(two * pi * z);
                    zj = -(tenth * std::cos(two * pi * x) * std::sin(two * pi * z));
                }
                T f[19];
                eup::equilibrium<T>(xj, yj, zj, f);
                const int64_t L = i + L2 * (j + M2 * (int64_t)k);
                for (int q = 0; q < 19; ++q) dst[q][L] = f[q];
            }
    }
}

}  // namespace

extern "C" {

int eup_init_reference(int32_t opt, int32_t l, int32_t m, int32_t n, const int32_t global[3], const int32_t start[3],
                       int32_t periodic, double u0, int32_t elem_bytes, void* const pops[19]) {
    if (!pops || !global || !start || (elem_bytes != 4 && elem_bytes != 8) || l < 1 || m < 1 || n < 1 ||
        global[0] < 1 || global[1] < 1 || global[2] < 1)
        return herr(EUP_ERR_INVALID_ARG, "eup_init_reference: bad argument");
    for (int q = 0; q < 19; ++q)
        if (!pops[q]) return herr(EUP_ERR_INVALID_ARG, "eup_init_reference: null population array");
    if (opt == 4 || opt == 5)
        return herr(EUP_ERR_UNSUPPORTED, "eup_init_reference: the reference stops on init option " +
                                              std::to_string(opt) + " (\"still to port\")");
    if (opt < 0 || opt > 5) return herr(EUP_ERR_INVALID_ARG, "eup_init_reference: option out of range [0,5]");
    if (elem_bytes == 4) init_reference_t<float>(opt, l, m, n, global, start, periodic != 0, u0, pops);
    else init_reference_t<double>(opt, l, m, n, global, start, periodic != 0, u0, pops);
    return EUP_OK;
}

int eup_init_equilibrium(int32_t l, int32_t m, int32_t n, double u_in, double amp, uint64_t seed, int32_t elem_bytes,
                         void* const pops[19]) {
    if (!pops || (elem_bytes != 4 && elem_bytes != 8) || l < 1 || m < 1 || n < 1)
        return herr(EUP_ERR_INVALID_ARG, "eup_init_equilibrium: bad argument");
    for (int q = 0; q < 19; ++q)
        if (!pops[q]) return herr(EUP_ERR_INVALID_ARG, "eup_init_equilibrium: null population array");
    if (elem_bytes == 4) init_state<float>(l, m, n, u_in, amp, seed, pops);
    else init_state<double>(l, m, n, u_in, amp, seed, pops);
    return EUP_OK;
}

int eup_geometry_reference(int32_t flag2, int32_t lx, int32_t ly, int32_t lz, int32_t variant, eup_geometry* g) {
    if (!g || lx < 1 || ly < 1 || lz < 1 || (variant & ~(EUP_GEOM_VARIANT_CYLINDER_INF | EUP_GEOM_VARIANT_TEST1)))
        return herr(EUP_ERR_INVALID_ARG, "eup_geometry_reference: bad argument");
    *g = eup_geometry{};
    int32_t radius = 0;
    // CODE/SRC/build.obs.F90:207-229 (sphere), :271-303 (column), :370-381 (half column)
    if (flag2 == 1) {
        g->kind = EUP_GEOM_REF_SPHERE;
        g->center[0] = lx / 4; g->center[1] = ly / 2; g->center[2] = lz / 2;
        radius = (variant & EUP_GEOM_VARIANT_TEST1) ? std::min(ly / 4, lz / 4) : 20;
        g->r2_lo = (int64_t)(radius - 2) * (radius - 2);
        g->r2_hi = (int64_t)(radius + 2) * (radius + 2);
        return EUP_OK;
    }
    if (flag2 == 2 || flag2 == 3) {
        g->kind = EUP_GEOM_REF_COLUMN;
        g->center[0] = lx / 4; g->center[1] = ly / 2; g->center[2] = 0;
        if (flag2 == 2 && (variant & EUP_GEOM_VARIANT_CYLINDER_INF)) {
            radius = 100;
            g->kstop = lz + 1;
        } else if (flag2 == 2) {
            radius = std::min(20, lx / 8);
            g->kstop = lz;  // sizeZ = lz from startZ = 0: the top layer k = lz stays fluid
        } else {
            radius = std::min(20, lz / 8);
            g->kstop = 60;
        }
        g->r2_lo = 0;
        g->r2_hi = (int64_t)(radius + 2) * (radius + 2);
        return EUP_OK;
    }
    return herr(EUP_ERR_UNSUPPORTED, "eup_geometry_reference: flag2 must be 1 (sphere), 2 (column) or 3 (half column)");
}

// The voxelisers' atan2 (geometry.h), exported for its accuracy test; not part of eup.h.
double eup_internal_atan2_det(double y, double x) { return eup::atan2_det(y, x); }

int eup_voxelise(const eup_geometry* g, int32_t l, int32_t m, int32_t n, int32_t* obs) {
    if (!g || !obs || l < 1 || m < 1 || n < 1) return herr(EUP_ERR_INVALID_ARG, "eup_voxelise: bad argument");
    eup::VoxShape S;
    std::vector<double> pores;
    std::string why;
    if (!eup::prepare_shape(*g, &S, &pores, &why)) return herr(EUP_ERR_INVALID_ARG, "eup_voxelise: " + why);
    S.ridge.pores = pores.data();
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t row = 0; row < (int64_t)m * n; ++row) {
        const int64_t gj = row % m + 1 + S.off[1], gk = row / m + 1 + S.off[2];
        int32_t* o = obs + row * l;
        for (int32_t i = 1; i <= l; ++i) o[i - 1] = eup::vox_solid(S, i + (int64_t)S.off[0], gj, gk) ? 1 : 0;
    }
    return EUP_OK;
}

int eup_geometry_cylinder_z(int32_t l, int32_t m, int32_t n, double xc, double yc, double r, int32_t* obs) {
    if (!obs || l < 1 || m < 1 || n < 1 || !(r >= 0)) return herr(EUP_ERR_INVALID_ARG, "eup_geometry_cylinder_z: bad argument");
    eup_geometry g{};
    g.kind = EUP_GEOM_CYLINDER_Z;
    g.xc = xc; g.yc = yc; g.radius = r;
    return eup_voxelise(&g, l, m, n, obs);
}

namespace {
eup_geometry shell_geometry(int32_t kind, double x0, double length, double yc, double zc, double outer_d,
                            double strut_d, double pitch, uint64_t seed) {
    eup_geometry g{};
    g.kind = kind;
    g.x0 = x0; g.length = length; g.yc = yc; g.zc = zc;
    g.outer_d = outer_d; g.strut_d = strut_d; g.pitch = pitch; g.seed = seed;
    return g;
}
}  // namespace

int eup_geometry_ridged_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                              double outer_d, double strut_d, double pitch, double ridge_h, double ridge_t,
                              double cap_t, double pore_d, double smooth_w, uint64_t seed, double* ns, double* dns_dh) {
    if (!ns || l < 1 || m < 1 || n < 1) return herr(EUP_ERR_INVALID_ARG, "eup_geometry_ridged_shell: bad argument");
    eup_geometry g = shell_geometry(EUP_GEOM_RIDGED_SHELL, x0, length, yc, zc, outer_d, strut_d, pitch, seed);
    g.ridge_h = ridge_h; g.ridge_t = ridge_t; g.cap_t = cap_t; g.pore_d = pore_d;
    eup::VoxShape S;
    std::vector<double> pores;
    std::string why;
    if (!eup::prepare_shape(g, &S, &pores, &why))
        return herr(EUP_ERR_INVALID_ARG, "eup_geometry_ridged_shell: bad argument (" + why + ")");
    S.ridge.pores = pores.data();
    const eup::RidgeShape& R = S.ridge;
    const double w = smooth_w > 0 ? smooth_w : 0.0;
    const double rmax = R.Ro + ridge_h + 4.0 * w + 1.0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t row = 0; row < (int64_t)m * n; ++row) {
        const int32_t j = (int32_t)(row % m) + 1, k = (int32_t)(row / m) + 1;
        const double dy = j - yc, dz = k - zc;
        for (int32_t i = 1; i <= l; ++i) {
            const int64_t o = (int64_t)(i - 1) + (int64_t)l * row;
            double v = eup::shell_solid(S.shell, i, j, k) ? 1.0 : 0.0, dv = 0.0;
            const eup::RidgeHit hit = eup::ridge_test(R, i - x0, dy, dz, rmax);
            if (hit.cap) v = 1.0;
            // ridges: a step at Ro + ridge_h, or 0.5 (1 + tanh((Ro + h - r)/w)) with its h-derivative
            if (hit.ridge_band) {
                double rv, rd;
                if (w > 0) {
                    const double z = (R.Ro + ridge_h - hit.r) / w;
                    rv = 0.5 * (1.0 + std::tanh(z));
                    const double c = std::cosh(z);
                    rd = 0.5 / (w * c * c);
                } else {
                    rv = (hit.r <= R.Ro + ridge_h) ? 1.0 : 0.0;
                    rd = 0.0;
                }
                if (rv > v) {
                    v = rv;
                    dv = rd;
                }
            }
            ns[o] = v;
            if (dns_dh) dns_dh[o] = dv;
        }
    }
    return EUP_OK;
}

int eup_geometry_reticular_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                                 double outer_d, double strut_d, double pitch, uint64_t seed, int32_t* obs) {
    if (!obs || l < 1 || m < 1 || n < 1 || !(outer_d > strut_d) || !(strut_d > 0) || !(pitch > 0) || !(length > 0))
        return herr(EUP_ERR_INVALID_ARG, "eup_geometry_reticular_shell: bad argument");
    const eup_geometry g = shell_geometry(EUP_GEOM_RETICULAR_SHELL, x0, length, yc, zc, outer_d, strut_d, pitch, seed);
    return eup_voxelise(&g, l, m, n, obs);
}

}  // extern "C"

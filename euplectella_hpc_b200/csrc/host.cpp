// Host utilities of the C ABI (no GPU): the reference's binary file formats,
// the synthetic initial state and the synthetic geometries.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/eup.h"
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

inline double wrap_pos(double a, double period) {
    double r = std::fmod(a, period);
    return r < 0 ? r + period : r;
}

// distance from point (u,s) to segment (u0,s0)-(u1,s1)
inline double seg_dist(double u, double s, double u0, double s0, double u1, double s1) {
    const double du = u1 - u0, ds = s1 - s0;
    double t = ((u - u0) * du + (s - s0) * ds) / (du * du + ds * ds);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const double eu = u - (u0 + t * du), es = s - (s0 + t * ds);
    return std::sqrt(eu * eu + es * es);
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

int eup_geometry_cylinder_z(int32_t l, int32_t m, int32_t n, double xc, double yc, double r, int32_t* obs) {
    if (!obs || l < 1 || m < 1 || n < 1 || !(r >= 0)) return herr(EUP_ERR_INVALID_ARG, "eup_geometry_cylinder_z: bad argument");
    for (int32_t k = 1; k <= n; ++k)
        for (int32_t j = 1; j <= m; ++j)
            for (int32_t i = 1; i <= l; ++i) {
                const double dx = i - xc, dy = j - yc;
                obs[(int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1))] = (dx * dx + dy * dy <= r * r) ? 1 : 0;
            }
    return EUP_OK;
}

int eup_geometry_ridged_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                              double outer_d, double strut_d, double pitch, double ridge_h, double ridge_t,
                              double cap_t, double pore_d, double smooth_w, uint64_t seed, double* ns, double* dns_dh) {
    if (!ns || l < 1 || m < 1 || n < 1 || !(ridge_h >= 0) || !(ridge_t > 0) || !(cap_t >= 0) || !(pore_d > 0))
        return herr(EUP_ERR_INVALID_ARG, "eup_geometry_ridged_shell: bad argument");
    const int64_t N = (int64_t)l * m * n;
    std::vector<int32_t> shell((size_t)N);
    int rc = eup_geometry_reticular_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, seed, shell.data());
    if (rc != EUP_OK) return rc;
    const double PI = 3.14159265358979323846;
    const double Ro = 0.5 * outer_d;            // outer surface of the shell
    const double period = 2.0 * PI * Ro;        // unrolled circumference at the outer surface
    const double phase = period * ((double)(splitmix64(seed ^ 0xA5A5A5A5ull) >> 11) * (1.0 / 9007199254740992.0));
    // porous cap: pores of diameter pore_d on a square grid of pitch 2*pore_d, each
    // centre jittered by up to pore_d/4 (seeded), kept if the pore fits inside r < Ro - 2
    std::vector<double> py, pz;
    const double cp = 2.0 * pore_d;
    int cnt = 0;
    for (double a = -Ro; a <= Ro; a += cp)
        for (double b = -Ro; b <= Ro; b += cp, ++cnt) {
            const uint64_t h1 = splitmix64(seed + 7919ull * (uint64_t)cnt), h2 = splitmix64(h1);
            const double ja = a + 0.25 * pore_d * (2.0 * ((double)(h1 >> 11) / 9007199254740992.0) - 1.0);
            const double jb = b + 0.25 * pore_d * (2.0 * ((double)(h2 >> 11) / 9007199254740992.0) - 1.0);
            if (std::sqrt(ja * ja + jb * jb) + 0.5 * pore_d < Ro - 2.0) {
                py.push_back(ja);
                pz.push_back(jb);
            }
        }
    const double w = smooth_w > 0 ? smooth_w : 0.0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t k = 1; k <= n; ++k)
        for (int32_t j = 1; j <= m; ++j) {
            const double dy = j - yc, dz = k - zc;
            const double r = std::sqrt(dy * dy + dz * dz);
            const double s = wrap_pos(Ro * std::atan2(dz, dy) - phase, period);
            for (int32_t i = 1; i <= l; ++i) {
                const int64_t o = (int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1));
                double v = shell[(size_t)o] ? 1.0 : 0.0, dv = 0.0;
                const double u = i - x0;
                // cap: the last cap_t of the shell's length, r < Ro, minus the pores
                if (u >= length - cap_t && u <= length && r < Ro) {
                    bool pore = false;
                    for (size_t p = 0; p < py.size() && !pore; ++p) {
                        const double ey = dy - py[p], ez = dz - pz[p];
                        pore = ey * ey + ez * ez <= 0.25 * pore_d * pore_d;
                    }
                    if (!pore) v = 1.0;
                }
                // two helical ridges at +-45 degrees on the outer surface: band of width
                // ridge_t about s = +-u (mod circumference), radially from Ro to Ro + h
                if (u >= 0 && u <= length && r > Ro - 1.0 && r < Ro + ridge_h + 4.0 * w + 1.0) {
                    double dperp = 1e30;
                    for (int sg = -1; sg <= 1; sg += 2) {
                        double d = wrap_pos(s - sg * u, period);
                        d = std::fmin(d, period - d) / std::sqrt(2.0);
                        dperp = std::fmin(dperp, d);
                    }
                    if (dperp <= 0.5 * ridge_t && r >= Ro - 0.5) {
                        double rv, rd;
                        if (w > 0) {
                            const double z = (Ro + ridge_h - r) / w;
                            rv = 0.5 * (1.0 + std::tanh(z));
                            const double c = std::cosh(z);
                            rd = 0.5 / (w * c * c);
                        } else {
                            rv = (r <= Ro + ridge_h) ? 1.0 : 0.0;
                            rd = 0.0;
                        }
                        if (rv > v) {
                            v = rv;
                            dv = rd;
                        }
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
    const double PI = 3.14159265358979323846;
    const double rs = 0.5 * strut_d;
    const double Rc = 0.5 * outer_d - rs;                 // strut centreline radius
    int ntheta = (int)std::lround(2.0 * PI * Rc / pitch);
    if (ntheta < 3) ntheta = 3;
    const double period = 2.0 * PI * Rc;                  // unrolled circumference
    const double ps = period / ntheta;                    // arc pitch
    const int ncell = (int)std::lround(length / pitch);   // cells along x
    const double ulen = ncell * pitch;
    const double phase = ps * ((double)(splitmix64(seed) >> 11) * (1.0 / 9007199254740992.0));
    std::memset(obs, 0, sizeof(int32_t) * (size_t)l * m * n);
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t k = 1; k <= n; ++k)
        for (int32_t j = 1; j <= m; ++j) {
            const double dy = j - yc, dz = k - zc;
            const double r = std::sqrt(dy * dy + dz * dz);
            const double dr = r - Rc;
            if (std::fabs(dr) > rs) continue;
            const double s = wrap_pos(Rc * std::atan2(dz, dy) - phase, period);
            const int b = (int)std::floor(s / ps);
            for (int32_t i = 1; i <= l; ++i) {
                const double u = i - x0;
                if (u < -rs || u > ulen + rs) continue;
                // longitudinal struts s = b*ps, running u in [0, ulen]
                const double uc = u < 0 ? 0 : (u > ulen ? ulen : u);
                const double ds_l = std::fmin(s - b * ps, (b + 1) * ps - s);
                double d = std::sqrt(ds_l * ds_l + (u - uc) * (u - uc));
                // rings u = a*pitch, a = 0..ncell
                int a = (int)std::lround(u / pitch);
                a = a < 0 ? 0 : (a > ncell ? ncell : a);
                d = std::fmin(d, std::fabs(u - a * pitch));
                // both diagonals of the cells with (ca + cb) even
                const int ca0 = (int)std::floor(u / pitch);
                for (int ca = ca0 - 1; ca <= ca0 + 1; ++ca) {
                    if (ca < 0 || ca >= ncell) continue;
                    for (int cb = b - 1; cb <= b + 1; ++cb) {
                        const int cbw = ((cb % ntheta) + ntheta) % ntheta;
                        if (((ca + cbw) & 1) != 0) continue;
                        const double u0 = ca * pitch, s0 = cb * ps;
                        d = std::fmin(d, seg_dist(u, s, u0, s0, u0 + pitch, s0 + ps));
                        d = std::fmin(d, seg_dist(u, s, u0, s0 + ps, u0 + pitch, s0));
                    }
                }
                if (dr * dr + d * d <= rs * rs)
                    obs[(int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1))] = 1;
            }
        }
    return EUP_OK;
}

}  // extern "C"

// Voxel geometries, evaluated node by node by the same code on the host
// (eup_voxelise and the eup_geometry_* helpers, OpenMP) and on the device
// (eup_build_obstacles, one warp per 32-bit mask word), so that both produce
// the same mask bit for bit.
//
// Only operations that IEEE 754 rounds correctly, or that are exact, appear in
// the node tests: + - * / and sqrt (correctly rounded on both sides; neither
// side contracts a multiply and an add: the device code is compiled with
// --fmad=false, the host code with -ffp-contract=off), floor, lround, fabs,
// fmin, fmod and integer arithmetic.  The angle about the shell axis needs atan2,
// which neither libm nor the CUDA math library rounds correctly, so the two
// could disagree on a voxel whose angle sits on a strut edge; atan2_det below
// computes it with basic operations only and therefore gives the same bits on
// both sides.
//
// Shapes (coordinates are global node indices: local (i, j, k) plus offset):
//   EUP_GEOM_REF_SPHERE, EUP_GEOM_REF_COLUMN  the obstacles CODE/SRC/build.obs.F90
//        creates (flag1 = 2): a spherical shell (flag2 = 1, :207-268) and a
//        z-column (flag2 = 2, :271-367; the half column of flag2 = 3, :370-441,
//        is a column with a shorter z extent);
//   EUP_GEOM_CYLINDER_Z     solid circular cylinder along z;
//   EUP_GEOM_RETICULAR_SHELL, EUP_GEOM_RIDGED_SHELL  the Euplectella-like lattice
//        shells of the synthetic workloads.
#pragma once
#include <math.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

#include "eup.h"
#include "init_eq.h"  // EUP_HD, splitmix64

namespace eup {

// ---- atan2 from basic operations -------------------------------------------

// atan(t) for 0 <= t <= 1 by the Maclaurin series atan t = sum_k (-1)^k t^(2k+1)/(2k+1)
// (Abramowitz & Stegun 4.4.42) after the reduction, for t > tan(pi/12) = 2 - sqrt3,
// atan t = pi/6 + atan((sqrt3 t - 1) / (sqrt3 + t)) (the tangent subtraction formula
// with tan(pi/6) = 1/sqrt3), which leaves |t| <= 2 - sqrt3; there t^2 < 0.0718 and 14
// terms bring the truncation below 2^-53 relative.  Within 2 ulp of libm's atan2.
EUP_HD inline double atan_unit(double t) {
    const double kSqrt3 = 1.7320508075688772935;
    const double kPi6 = 0.52359877559829887308;
    const double kTanPi12 = 0.26794919243112270647;
    double base = 0.0;
    if (t > kTanPi12) {
        t = (kSqrt3 * t - 1.0) / (kSqrt3 + t);
        base = kPi6;
    }
    const double t2 = t * t;
    double s = 0.0;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int k = 13; k >= 0; --k) s = 1.0 / (double)(2 * k + 1) - t2 * s;
    return base + t * s;
}

// Angle of (x, y) in [-pi, pi], signed like y (a negative zero included); 0 at the origin.
EUP_HD inline double atan2_det(double y, double x) {
    const double kPi2 = 1.5707963267948966192, kPi = 3.1415926535897932385;
    const double ax = fabs(x), ay = fabs(y);
    if (ax == 0.0 && ay == 0.0) return 0.0;
    const bool swap = ay > ax;
    double a = atan_unit(swap ? ax / ay : ay / ax);
    if (swap) a = kPi2 - a;
    if (x < 0.0) a = kPi - a;
    if (signbit(y)) a = -a;
    return a;
}

EUP_HD inline double wrap_pos(double a, double period) {
    const double r = fmod(a, period);
    return r < 0 ? r + period : r;
}

// distance from point (u,s) to segment (u0,s0)-(u1,s1)
EUP_HD inline double seg_dist(double u, double s, double u0, double s0, double u1, double s1) {
    const double du = u1 - u0, ds = s1 - s0;
    double t = ((u - u0) * du + (s - s0) * ds) / (du * du + ds * ds);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const double eu = u - (u0 + t * du), es = s - (s0 + t * ds);
    return sqrt(eu * eu + es * es);
}

// ---- shape parameters, derived once on the host ------------------------------

struct RefShape {        // EUP_GEOM_REF_SPHERE / EUP_GEOM_REF_COLUMN
    int32_t ic, jc, kc;  // integer centre (global)
    int64_t r2_lo, r2_hi;
    int32_t kstop;       // column: global k < kstop
};

struct ShellShape {      // reticular shell (axis x)
    double x0, yc, zc;
    double rs, Rc;       // strut radius, strut centreline radius
    double period, ps;   // unrolled circumference at Rc, arc pitch
    double pitch, ulen, phase;
    int32_t ntheta, ncell;
};

struct RidgeShape {      // ridges and porous cap of the ridged shell
    double Ro, period, phase;
    double length, cap_t, pore_r2, ridge_h, ridge_t;
    int32_t npores;
    const double* pores;  // npores (y, z) centres relative to the axis
};

struct VoxShape {
    int32_t kind;
    int32_t off[3];
    RefShape ref;
    double xc, yc, r2;    // cylinder_z
    ShellShape shell;
    RidgeShape ridge;
};

// ---- node tests ------------------------------------------------------------

// CODE/SRC/build.obs.F90:238-245 (sphere) and :331-339 (column).  The reference
// forms d2 in integer arithmetic, stores it in a real and compares it with the
// reals (R -+ 2)^2; with an integer radius below 4094 those bounds are exact
// integers in single precision and rounding is monotone, so comparing the
// integers themselves gives the same answer.
EUP_HD inline bool ref_solid(const VoxShape& S, int64_t gi, int64_t gj, int64_t gk) {
    const RefShape& R = S.ref;
    const int64_t di = R.ic - gi, dj = R.jc - gj;
    if (S.kind == EUP_GEOM_REF_SPHERE) {
        const int64_t dk = R.kc - gk;
        const int64_t d2 = di * di + dj * dj + dk * dk;
        return d2 > R.r2_lo && d2 < R.r2_hi;
    }
    // column: startZ = kcoord - mpicoords(3) n, stopZ = startZ + sizeZ, k in [startZ, stopZ)
    if (gk < R.kc || gk >= R.kstop) return false;
    const int64_t d2 = di * di + dj * dj;
    return d2 >= R.r2_lo && d2 < R.r2_hi;
}

// Distance-based test of the reticular shell at column (r, s, b) and axial position u.
EUP_HD inline bool shell_solid_at(const ShellShape& P, double dr, double s, int b, double u) {
    const double rs = P.rs, pitch = P.pitch, ps = P.ps, ulen = P.ulen;
    if (u < -rs || u > ulen + rs) return false;
    // longitudinal struts s = b*ps, running u in [0, ulen]
    const double uc = u < 0 ? 0 : (u > ulen ? ulen : u);
    const double ds_l = fmin(s - b * ps, (b + 1) * ps - s);
    double d = sqrt(ds_l * ds_l + (u - uc) * (u - uc));
    // rings u = a*pitch, a = 0..ncell
    int a = (int)lround(u / pitch);
    a = a < 0 ? 0 : (a > P.ncell ? P.ncell : a);
    d = fmin(d, fabs(u - a * pitch));
    // both diagonals of the cells with (ca + cb) even
    const int ca0 = (int)floor(u / pitch);
    for (int ca = ca0 - 1; ca <= ca0 + 1; ++ca) {
        if (ca < 0 || ca >= P.ncell) continue;
        for (int cb = b - 1; cb <= b + 1; ++cb) {
            const int cbw = ((cb % P.ntheta) + P.ntheta) % P.ntheta;
            if (((ca + cbw) & 1) != 0) continue;
            const double u0 = ca * pitch, s0 = cb * ps;
            d = fmin(d, seg_dist(u, s, u0, s0, u0 + pitch, s0 + ps));
            d = fmin(d, seg_dist(u, s, u0, s0 + ps, u0 + pitch, s0));
        }
    }
    return dr * dr + d * d <= rs * rs;
}

EUP_HD inline bool shell_solid(const ShellShape& P, double gi, double gj, double gk) {
    const double dy = gj - P.yc, dz = gk - P.zc;
    const double r = sqrt(dy * dy + dz * dz);
    const double dr = r - P.Rc;
    if (fabs(dr) > P.rs) return false;
    const double s = wrap_pos(P.Rc * atan2_det(dz, dy) - P.phase, P.period);
    const int b = (int)floor(s / P.ps);
    return shell_solid_at(P, dr, s, b, gi - P.x0);
}

// Cap and ridge tests of the ridged shell at one node.  cap: inside the last cap_t of
// the shell's length at r < Ro and outside every pore.  ridge: inside the band of width
// ridge_t about either +-45 degree helix s = +-u on the outer surface, at r >= Ro - 1/2;
// the caller applies the radial profile (a step at Ro + ridge_h, or its smoothing).
struct RidgeHit {
    bool cap, ridge_band;
    double r;
};

EUP_HD inline RidgeHit ridge_test(const RidgeShape& P, double u, double dy, double dz, double rmax) {
    RidgeHit h{false, false, 0.0};
    const double r = sqrt(dy * dy + dz * dz);
    h.r = r;
    if (u >= P.length - P.cap_t && u <= P.length && r < P.Ro) {
        bool pore = false;
        for (int p = 0; p < P.npores && !pore; ++p) {
            const double ey = dy - P.pores[2 * p], ez = dz - P.pores[2 * p + 1];
            pore = ey * ey + ez * ez <= P.pore_r2;
        }
        h.cap = !pore;
    }
    if (u >= 0 && u <= P.length && r > P.Ro - 1.0 && r < rmax) {
        const double s = wrap_pos(P.Ro * atan2_det(dz, dy) - P.phase, P.period);
        double dperp = 1e30;
        for (int sg = -1; sg <= 1; sg += 2) {
            double d = wrap_pos(s - sg * u, P.period);
            d = fmin(d, P.period - d) / sqrt(2.0);
            dperp = fmin(dperp, d);
        }
        h.ridge_band = dperp <= 0.5 * P.ridge_t && r >= P.Ro - 0.5;
    }
    return h;
}

// The 0/1 obstacle of shape S at global node (gi, gj, gk).
EUP_HD inline bool vox_solid(const VoxShape& S, int64_t gi, int64_t gj, int64_t gk) {
    switch (S.kind) {
        case EUP_GEOM_REF_SPHERE:
        case EUP_GEOM_REF_COLUMN:
            return ref_solid(S, gi, gj, gk);
        case EUP_GEOM_CYLINDER_Z: {
            const double dx = (double)gi - S.xc, dy = (double)gj - S.yc;
            return dx * dx + dy * dy <= S.r2;
        }
        case EUP_GEOM_RETICULAR_SHELL:
            return shell_solid(S.shell, (double)gi, (double)gj, (double)gk);
        case EUP_GEOM_RIDGED_SHELL: {
            if (shell_solid(S.shell, (double)gi, (double)gj, (double)gk)) return true;
            const RidgeShape& P = S.ridge;
            const double dy = (double)gj - S.shell.yc, dz = (double)gk - S.shell.zc;
            const RidgeHit h = ridge_test(P, (double)gi - S.shell.x0, dy, dz, P.Ro + P.ridge_h + 1.0);
            return h.cap || (h.ridge_band && h.r <= P.Ro + P.ridge_h);
        }
        default:
            return false;
    }
}

// ---- parameters of a shape, derived once on the host --------------------------

// Fills S from g; the cap pores of a ridged shell go to *pores ((y, z) pairs; S.ridge.pores
// is left for the caller to point at host or device storage).  False with *why on a bad shape.
inline bool prepare_shape(const eup_geometry& g, VoxShape* S, std::vector<double>* pores, std::string* why) {
    const double PI = 3.14159265358979323846;
    *S = VoxShape{};
    S->kind = g.kind;
    for (int d = 0; d < 3; ++d) S->off[d] = g.offset[d];
    pores->clear();
    switch (g.kind) {
        case EUP_GEOM_NONE:
            return true;
        case EUP_GEOM_REF_SPHERE:
        case EUP_GEOM_REF_COLUMN:
            if (g.r2_lo < 0 || g.r2_hi < g.r2_lo) { *why = "r2_lo/r2_hi out of order"; return false; }
            S->ref = RefShape{g.center[0], g.center[1], g.center[2], g.r2_lo, g.r2_hi, g.kstop};
            return true;
        case EUP_GEOM_CYLINDER_Z:
            if (!(g.radius >= 0)) { *why = "negative radius"; return false; }
            S->xc = g.xc;
            S->yc = g.yc;
            S->r2 = g.radius * g.radius;
            return true;
        case EUP_GEOM_RETICULAR_SHELL:
        case EUP_GEOM_RIDGED_SHELL: {
            if (!(g.outer_d > g.strut_d) || !(g.strut_d > 0) || !(g.pitch > 0) || !(g.length > 0)) {
                *why = "shell needs outer_d > strut_d > 0, pitch > 0, length > 0";
                return false;
            }
            ShellShape& P = S->shell;
            P.x0 = g.x0;
            P.yc = g.yc;
            P.zc = g.zc;
            P.rs = 0.5 * g.strut_d;
            P.Rc = 0.5 * g.outer_d - P.rs;                      // strut centreline radius
            int ntheta = (int)std::lround(2.0 * PI * P.Rc / g.pitch);
            P.ntheta = ntheta < 3 ? 3 : ntheta;
            P.period = 2.0 * PI * P.Rc;                          // unrolled circumference
            P.ps = P.period / P.ntheta;                          // arc pitch
            P.pitch = g.pitch;
            P.ncell = (int)std::lround(g.length / g.pitch);      // cells along x
            P.ulen = P.ncell * g.pitch;
            P.phase = P.ps * ((double)(splitmix64(g.seed) >> 11) * (1.0 / 9007199254740992.0));
            if (g.kind == EUP_GEOM_RETICULAR_SHELL) return true;
            if (!(g.ridge_h >= 0) || !(g.ridge_t > 0) || !(g.cap_t >= 0) || !(g.pore_d > 0)) {
                *why = "ridged shell needs ridge_h >= 0, ridge_t > 0, cap_t >= 0, pore_d > 0";
                return false;
            }
            RidgeShape& R = S->ridge;
            R.Ro = 0.5 * g.outer_d;                              // outer surface of the shell
            R.period = 2.0 * PI * R.Ro;                          // unrolled circumference there
            R.phase = R.period * ((double)(splitmix64(g.seed ^ 0xA5A5A5A5ull) >> 11) * (1.0 / 9007199254740992.0));
            R.length = g.length;
            R.cap_t = g.cap_t;
            R.pore_r2 = 0.25 * g.pore_d * g.pore_d;
            R.ridge_h = g.ridge_h;
            R.ridge_t = g.ridge_t;
            // porous cap: pores of diameter pore_d on a square grid of pitch 2*pore_d, each
            // centre jittered by up to pore_d/4 (seeded), kept if the pore fits inside r < Ro - 2
            const double cp = 2.0 * g.pore_d;
            int cnt = 0;
            for (double a = -R.Ro; a <= R.Ro; a += cp)
                for (double b = -R.Ro; b <= R.Ro; b += cp, ++cnt) {
                    const uint64_t h1 = splitmix64(g.seed + 7919ull * (uint64_t)cnt), h2 = splitmix64(h1);
                    const double ja = a + 0.25 * g.pore_d * (2.0 * ((double)(h1 >> 11) / 9007199254740992.0) - 1.0);
                    const double jb = b + 0.25 * g.pore_d * (2.0 * ((double)(h2 >> 11) / 9007199254740992.0) - 1.0);
                    if (std::sqrt(ja * ja + jb * jb) + 0.5 * g.pore_d < R.Ro - 2.0) {
                        pores->push_back(ja);
                        pores->push_back(jb);
                    }
                }
            R.npores = (int32_t)(pores->size() / 2);
            return true;
        }
        default:
            *why = "unknown geometry kind " + std::to_string(g.kind);
            return false;
    }
}

}  // namespace eup

/*
 * oracle/orc_geom.c -- CPU ORACLE (test infrastructure only; see orc.h):
 * the synthetic bodies of the benchmark workloads, voxelised on the host so
 * that the CPU baseline and the reference arm of the benchmark build their
 * input without the product library.
 *
 * The reference ships no geometry for these sizes (its production obstacles
 * are unshipped files read by CODE/SRC/build.obs.F90:147-177), so these
 * bodies are definitions of the workload, not restatements of reference code:
 *   - a solid circular cylinder along z:  (i - xc)^2 + (j - yc)^2 <= r^2;
 *   - the reticular cylindrical shell (axis x): struts of radius rs whose
 *     centrelines lie on the cylinder of radius Rc = outer_d/2 - rs, unrolled
 *     into the plane (u = x - x0 along the axis, s = arc length about it):
 *     longitudinal struts at s = b*ps (ntheta of them, ps = 2 pi Rc / ntheta,
 *     ntheta = round(2 pi Rc / pitch)), rings at u = a*pitch (a = 0..ncell,
 *     ncell = round(length / pitch)), and both diagonals of every cell
 *     (a, b) with a + b even; a node is solid when its distance to the
 *     nearest strut centreline, measured in (radial offset, unrolled
 *     distance), is at most rs.  The angle origin is turned by a seeded
 *     phase (splitmix64 of the seed).
 * The arithmetic uses only operations IEEE 754 rounds correctly (+ - * /,
 * sqrt) or exact ones, compiled without contraction, and an atan2 built from
 * them (octant reduction, the tangent subtraction formula with
 * tan(pi/6) = 1/sqrt3 down to |t| <= tan(pi/12), then 14 terms of the
 * Maclaurin series of atan), so the mask is the same bit for bit on every
 * IEEE machine, the product's device and host voxelisers included (tested).
 */
#include <math.h>
#include <stdint.h>

#include "orc.h"

static double orc_atan_unit(double t)
{
    const double sqrt3 = 1.7320508075688772935, pi6 = 0.52359877559829887308;
    const double tan_pi12 = 0.26794919243112270647;
    double base = 0.0;
    if (t > tan_pi12) {
        t = (sqrt3 * t - 1.0) / (sqrt3 + t);
        base = pi6;
    }
    const double t2 = t * t;
    double s = 0.0;
    for (int k = 13; k >= 0; --k) s = 1.0 / (double)(2 * k + 1) - t2 * s;
    return base + t * s;
}

/* angle of (x, y) in [-pi, pi], signed like y; 0 at the origin */
static double orc_atan2(double y, double x)
{
    const double pi2 = 1.5707963267948966192, pi = 3.1415926535897932385;
    const double ax = fabs(x), ay = fabs(y);
    if (ax == 0.0 && ay == 0.0) return 0.0;
    const int steep = ay > ax;
    double a = orc_atan_unit(steep ? ax / ay : ay / ax);
    if (steep) a = pi2 - a;
    if (x < 0.0) a = pi - a;
    if (signbit(y)) a = -a;
    return a;
}

static double orc_wrap(double a, double period)
{
    const double r = fmod(a, period);
    return r < 0 ? r + period : r;
}

/* distance from (u, s) to the segment (u0, s0)-(u1, s1) */
static double orc_seg(double u, double s, double u0, double s0, double u1, double s1)
{
    const double du = u1 - u0, ds = s1 - s0;
    double t = ((u - u0) * du + (s - s0) * ds) / (du * du + ds * ds);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const double eu = u - (u0 + t * du), es = s - (s0 + t * ds);
    return sqrt(eu * eu + es * es);
}

typedef struct {
    double x0, yc, zc, rs, Rc, period, ps, pitch, ulen, phase;
    int ntheta, ncell;
} orc_shell;

static orc_shell orc_shell_make(double x0, double length, double yc, double zc, double outer_d, double strut_d,
                                double pitch, uint64_t seed)
{
    const double pi = 3.14159265358979323846;
    orc_shell P;
    P.x0 = x0;
    P.yc = yc;
    P.zc = zc;
    P.rs = 0.5 * strut_d;
    P.Rc = 0.5 * outer_d - P.rs;
    P.ntheta = (int)lround(2.0 * pi * P.Rc / pitch);
    if (P.ntheta < 3) P.ntheta = 3;
    P.period = 2.0 * pi * P.Rc;
    P.ps = P.period / P.ntheta;
    P.pitch = pitch;
    P.ncell = (int)lround(length / pitch);
    P.ulen = P.ncell * pitch;
    P.phase = P.ps * ((double)(orc_splitmix64(seed) >> 11) * (1.0 / 9007199254740992.0));
    return P;
}

static int orc_shell_solid(const orc_shell* P, double gi, double gj, double gk)
{
    const double dy = gj - P->yc, dz = gk - P->zc;
    const double r = sqrt(dy * dy + dz * dz);
    const double dr = r - P->Rc;
    if (fabs(dr) > P->rs) return 0;
    const double s = orc_wrap(P->Rc * orc_atan2(dz, dy) - P->phase, P->period);
    const int b = (int)floor(s / P->ps);
    const double u = gi - P->x0;
    const double rs = P->rs, pitch = P->pitch, ps = P->ps, ulen = P->ulen;
    if (u < -rs || u > ulen + rs) return 0;
    /* longitudinal struts (their u-extent is [0, ulen]) */
    const double uc = u < 0 ? 0 : (u > ulen ? ulen : u);
    const double ds_l = fmin(s - b * ps, (b + 1) * ps - s);
    double d = sqrt(ds_l * ds_l + (u - uc) * (u - uc));
    /* nearest ring */
    int a = (int)lround(u / pitch);
    a = a < 0 ? 0 : (a > P->ncell ? P->ncell : a);
    d = fmin(d, fabs(u - a * pitch));
    /* diagonals of the neighbouring cells with (ca + cb) even */
    const int ca0 = (int)floor(u / pitch);
    for (int ca = ca0 - 1; ca <= ca0 + 1; ++ca) {
        if (ca < 0 || ca >= P->ncell) continue;
        for (int cb = b - 1; cb <= b + 1; ++cb) {
            const int cbw = ((cb % P->ntheta) + P->ntheta) % P->ntheta;
            if (((ca + cbw) & 1) != 0) continue;
            const double u0 = ca * pitch, s0 = cb * ps;
            d = fmin(d, orc_seg(u, s, u0, s0, u0 + pitch, s0 + ps));
            d = fmin(d, orc_seg(u, s, u0, s0 + ps, u0 + pitch, s0));
        }
    }
    return dr * dr + d * d <= rs * rs;
}

int64_t orc_voxelise_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                           double outer_d, double strut_d, double pitch, uint64_t seed, int32_t* obs)
{
    const orc_shell P = orc_shell_make(x0, length, yc, zc, outer_d, strut_d, pitch, seed);
    int64_t cnt = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : cnt)
    for (int64_t row = 0; row < (int64_t)m * n; ++row) {
        const int j = (int)(row % m) + 1, k = (int)(row / m) + 1;
        int32_t* o = obs + row * l;
        for (int i = 1; i <= l; ++i) {
            o[i - 1] = orc_shell_solid(&P, (double)i, (double)j, (double)k);
            cnt += o[i - 1];
        }
    }
    return cnt;
}

int64_t orc_voxelise_cylinder_z(int32_t l, int32_t m, int32_t n, double xc, double yc, double r, int32_t* obs)
{
    const double r2 = r * r;
    int64_t cnt = 0;
#pragma omp parallel for schedule(static) reduction(+ : cnt)
    for (int64_t row = 0; row < (int64_t)m * n; ++row) {
        const int j = (int)(row % m) + 1;
        int32_t* o = obs + row * l;
        for (int i = 1; i <= l; ++i) {
            const double dx = (double)i - xc, dy = (double)j - yc;
            o[i - 1] = dx * dx + dy * dy <= r2;
            cnt += o[i - 1];
        }
    }
    return cnt;
}

// Device-side building blocks of the D3Q19 BGK step: lattice constants,
// population storage formats, the halo shell and the collision.
//
// Population q (0-based) is the reference's a(q+1); velocities follow
// CODE/SRC/bgk3d.F90:30-49 and the streaming offsets of CODE/SRC/movef.F90:48-65.
// All kernels of this library are compiled with --fmad=false: every float or
// double operation rounds on its own, in the evaluation order of the
// reference's Fortran, so the FP32 and FP64 paths reproduce a serial IEEE
// build of the reference bit for bit.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace eup {

constexpr int Q = 19;

// c_q, q = 0..18 (reference a01..a19)
__host__ __device__ constexpr int cx_of(int q) {
    return (q <= 4) ? 1 : (q >= 9 && q <= 13) ? -1 : 0;
}
__host__ __device__ constexpr int cy_of(int q) {
    return (q == 2 || q == 6 || q == 7 || q == 8 || q == 11) ? 1
           : (q == 0 || q == 9 || q == 15 || q == 16 || q == 17) ? -1
                                                                  : 0;
}
__host__ __device__ constexpr int cz_of(int q) {
    return (q == 3 || q == 5 || q == 6 || q == 12 || q == 17) ? 1
           : (q == 1 || q == 8 || q == 10 || q == 14 || q == 15) ? -1
                                                                  : 0;
}
// opposite direction: 1<->12, 2<->13, 3<->10, 4<->11, 5<->14, 6<->15, 7<->16, 8<->17, 9<->18
__host__ __device__ constexpr int opp_of(int q) {
    return (q == 18) ? 18 : (q <= 1) ? q + 11 : (q <= 3) ? q + 7 : (q <= 8) ? q + 9
           : (q <= 10) ? q - 7 : (q <= 12) ? q - 11 : q - 9;
}
// weight class: 0 -> p0 (rest), 1 -> p1 (axis), 2 -> p2 (diagonal)
__host__ __device__ constexpr int wclass_of(int q) {
    return (q == 18) ? 0 : (q == 4 || q == 5 || q == 7 || q == 13 || q == 14 || q == 16) ? 1 : 2;
}

template <typename R> struct Const;
template <> struct Const<float> {
    // CODE/SRC/storage.F90:54-81,194-205: computed wide, rounded to mykind
    static __device__ __forceinline__ float p0() { return (float)(1.0 / 3.0); }
    static __device__ __forceinline__ float p1() { return (float)(1.0 / 18.0); }
    static __device__ __forceinline__ float p2() { return (float)(1.0 / 36.0); }
};
template <> struct Const<double> {
    static __device__ __forceinline__ double p0() { return 1.0 / 3.0; }
    static __device__ __forceinline__ double p1() { return 1.0 / 18.0; }
    static __device__ __forceinline__ double p2() { return 1.0 / 36.0; }
};

// Two FP32 lanes operated on together with the packed FP32 instructions of
// sm_100 (add/mul/fma .f32x2).  Each lane is rounded exactly as the scalar
// operation, so code written once for R = float and R = F2 gives identical
// bits per lane; F2 lets one thread collide two nodes with half the FP32
// instructions.  Division has no packed form and runs per lane.
struct F2 {
    float2 v;
    F2() = default;
    __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit F2(float2 w) : v(w) {}
};
// Every packed operation is issued as a packed fused multiply-add: a product is
// fma(a, b, z) and a sum fma(a, u, b) with u = 1 and z = -0 read from constant
// memory, each exactly the correctly rounded product or sum.  The code
// generator fuses a packed multiply feeding a packed add into one fma (even
// with an explicit .rn rounding modifier), which would skip a rounding of the
// scalar reference-order arithmetic; with u and z unknown when the kernel is
// compiled no operation can be rewritten as a plain multiply or add, and an
// fma is never fused with another.
__constant__ float2 kF2Unit = {1.0f, -0.0f};

__device__ __forceinline__ F2 fma_rn(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return fma_rn(a, F2(kF2Unit.x), b); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(-a.v.x, -a.v.y); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return fma_rn(b, F2(-kF2Unit.x), a); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return fma_rn(a, b, F2(kF2Unit.y)); }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.v.x / b.v.x, a.v.y / b.v.y); }

template <> struct Const<F2> {
    static __device__ __forceinline__ F2 p0() { return F2(Const<float>::p0()); }
    static __device__ __forceinline__ F2 p1() { return F2(Const<float>::p1()); }
    static __device__ __forceinline__ F2 p2() { return F2(Const<float>::p2()); }
};

template <typename R>
__device__ __forceinline__ R weight(int q) {
    const int c = wclass_of(q);
    return c == 0 ? Const<R>::p0() : (c == 1 ? Const<R>::p1() : Const<R>::p2());
}

// ---------------------------------------------------------------------------
// Storage formats.  S is what lives in HBM, R the arithmetic type.
//   float/double : the population itself;
//   __half/bf16  : (f_q - w_q) * scale, scale a power of two.
// ---------------------------------------------------------------------------
template <typename S, typename R> struct Store;

template <> struct Store<float, float> {
    static __device__ __forceinline__ float load(float s, int, float) { return s; }
    static __device__ __forceinline__ float store(float f, int, float) { return f; }
};
template <> struct Store<double, double> {
    static __device__ __forceinline__ double load(double s, int, double) { return s; }
    static __device__ __forceinline__ double store(double f, int, double) { return f; }
};
template <> struct Store<__half, float> {
    static __device__ __forceinline__ float load(__half s, int q, float inv_scale) {
        return weight<float>(q) + __half2float(s) * inv_scale;
    }
    static __device__ __forceinline__ __half store(float f, int q, float scale) {
        return __float2half_rn((f - weight<float>(q)) * scale);
    }
};
template <> struct Store<__nv_bfloat16, float> {
    static __device__ __forceinline__ float load(__nv_bfloat16 s, int q, float inv_scale) {
        return weight<float>(q) + __bfloat162float(s) * inv_scale;
    }
    static __device__ __forceinline__ __nv_bfloat16 store(float f, int q, float scale) {
        return __float2bfloat16_rn((f - weight<float>(q)) * scale);
    }
};

// ---------------------------------------------------------------------------
// Lattice geometry and the persistent halo shell.
//
// Interior node (i,j,k), 1-based, lives at lin = (i-1) + l*((j-1) + m*(k-1))
// of each population array.  Halo nodes (any coordinate 0 or l+1/m+1/n+1)
// live in one shell per population with a single owner per node: the x
// planes own their full (m+2)*(n+2) extent, the y planes i = 1..l and
// k = 0..n+1, the z planes i = 1..l, j = 1..m.  The shell plays the role of
// the halo of the reference's single array a (CODE/SRC/alloca.F90:94-132):
// it persists across steps, so halo values that the reference never rewrites
// keep their initial values here too.
// ---------------------------------------------------------------------------
struct Geo {
    int l, m, n;
    int64_t lm;      // l*m
    int64_t N;       // l*m*n
    int64_t sx, sy, sz;         // face sizes
    int64_t ox0, oxl, oy0, oym, oz0, ozn, G;
    int64_t mn, xr, xs;  // m*n; one rim of the x-face copy; elements per side (18 m*n + 2 rims)

    __host__ __device__ void init(int l_, int m_, int n_) {
        l = l_; m = m_; n = n_;
        lm = (int64_t)l * m;
        N = lm * n;
        sx = (int64_t)(m + 2) * (n + 2);
        sy = (int64_t)l * (n + 2);
        sz = (int64_t)l * m;
        ox0 = 0; oxl = sx; oy0 = 2 * sx; oym = oy0 + sy; oz0 = oym + sy; ozn = oz0 + sz;
        G = ozn + sz;
        mn = (int64_t)m * n;
        xr = 5 * (2 * (int64_t)(m + 2) + 2 * (int64_t)n);
        xs = 18 * mn + 2 * xr;
    }
    __host__ __device__ __forceinline__ bool interior(int i, int j, int k) const {
        return i >= 1 && i <= l && j >= 1 && j <= m && k >= 1 && k <= n;
    }
    __host__ __device__ __forceinline__ int64_t lin(int i, int j, int k) const {
        return (int64_t)(i - 1) + (int64_t)l * ((int64_t)(j - 1) + (int64_t)m * (k - 1));
    }
    // (i,j,k) must be a halo node
    __host__ __device__ __forceinline__ int64_t gidx(int i, int j, int k) const {
        if (i == 0) return ox0 + (int64_t)k * (m + 2) + j;
        if (i == l + 1) return oxl + (int64_t)k * (m + 2) + j;
        if (j == 0) return oy0 + (int64_t)k * l + (i - 1);
        if (j == m + 1) return oym + (int64_t)k * l + (i - 1);
        if (k == 0) return oz0 + (int64_t)(j - 1) * l + (i - 1);
        return ozn + (int64_t)(j - 1) * l + (i - 1);
    }
};

// Row (j, k) of face row index f, 0 <= f < nz m + (n-2) ny (nz = 2 for n >= 2, else 1;
// ny = 2 for m >= 2, else 1): the rows on the y/z boundary planes, first the planes k = 1
// and k = n (all j), then j = 1 and j = m of the planes k = 2 .. n-1.
__host__ __device__ __forceinline__ void face_row(const Geo& g, int f, int* j, int* k) {
    const int nz = g.n >= 2 ? 2 : 1, ny = g.m >= 2 ? 2 : 1;
    if (f < nz * g.m) {
        *k = f < g.m ? 1 : g.n;
        *j = f % g.m + 1;
    } else {
        const int r = f - nz * g.m;
        *k = 2 + r / ny;
        *j = (r % ny == 0) ? 1 : g.m;
    }
}

// Pointers of one lattice (19 population arrays) plus the halo shell and the
// x-face copy.  The x-face copy holds, for the interior columns x = 1 (side 0)
// and x = l (side 1), the 18 moving populations exactly as a load from the
// lattice returns them.  The stream-collide kernel writes it for the state it
// produces and the bounce-back kernel keeps it in step, so that halo kernels
// read these columns coalesced in j instead of with a stride of l elements.
//
// Layout per side: a rim, 18 slots of m*n values ((j-1) + (k-1)*m), a second
// rim; each rim holds 5 * (2(m+2) + 2n) values and the two sides are one
// constant stride apart.  The slot order, the same on both sides, puts the
// five populations leaving through the x = 1 face (cx = -1, q 9..13) first and
// those leaving through x = l (cx = +1, q 0..4) last.  Side 0's first rim and
// side 1's second rim hold these populations on the face column's halo rows
// (k = 0 and k = n+1 for j = 0..m+1, then j = 0 and j = m+1 for k = 1..n),
// packed after the halo kernels of an x-slab step; the other two rims are
// unused.  So side 0's rim + slots 0..4 and side 1's slots 13..17 + rim are
// each one contiguous plane message of 5 (m+2)(n+2) values that the
// stream-collide epilogue has already written: the send buffers of the
// x-slab plane exchange, with no pack kernel over the plane.
template <typename S, typename R>
struct Lat {
    S* pop[Q];
    R* ghost;       // ghost[q*G + gidx]
    R* xface;       // [2][18 * m*n + rim]
    R scale, inv_scale;
};

// Slot of population q: q 9..13 -> 0..4, q 5..8 -> 5..8, q 14..17 -> 9..12, q 0..4 -> 13..17.
__host__ __device__ __forceinline__ constexpr int xface_slot(int q) {
    return q <= 4 ? q + 13 : (q >= 9 && q <= 13) ? q - 9 : (q <= 8 ? q : q - 5);
}
// Elements of the whole x-face copy (both sides).
__host__ __device__ __forceinline__ int64_t xface_elems(const Geo& g) { return 2 * g.xs; }
// Offset of side `side`'s plane message: side 0 = rim then q 9..13, side 1 = q 0..4 then rim.
__host__ __device__ __forceinline__ int64_t xface_send_offset(const Geo& g, int side) {
    return side ? g.xs + g.xr + 13 * g.mn : 0;
}
// Offset of the rim of side `side`'s plane message.
__host__ __device__ __forceinline__ int64_t xface_rim_offset(const Geo& g, int side) {
    return side ? g.xs + g.xr + 18 * g.mn : 0;
}
// Halo-row node (j, k) of the face plane at position p (0 <= p < 2(m+2) + 2n) of one
// population's rim.
__host__ __device__ __forceinline__ void xface_rim_node(const Geo& g, int64_t p, int* j, int* k) {
    if (p < 2 * (int64_t)(g.m + 2)) {
        *k = p < g.m + 2 ? 0 : g.n + 1;
        *j = (int)(p < g.m + 2 ? p : p - (g.m + 2));
    } else {
        const int64_t e = p - 2 * (int64_t)(g.m + 2);
        *j = e < g.n ? 0 : g.m + 1;
        *k = (int)(e < g.n ? e : e - g.n) + 1;
    }
}

template <typename S, typename R>
__device__ __forceinline__ R lat_load(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k) {
    if (g.interior(i, j, k)) return Store<S, R>::load(L.pop[q][g.lin(i, j, k)], q, L.inv_scale);
    return L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)];
}

__host__ __device__ __forceinline__ int64_t xface_idx(const Geo& g, int side, int q, int j, int k) {
    return side * g.xs + g.xr + (int64_t)xface_slot(q) * g.mn + (j - 1) + (int64_t)(k - 1) * g.m;
}

// Load used by the halo kernels: x-face columns from the x-face copy.
template <typename S, typename R>
__device__ __forceinline__ R bc_load(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k) {
    if (q < 18 && (i == 1 || i == g.l) && j >= 1 && j <= g.m && k >= 1 && k <= g.n)
        return L.xface[xface_idx(g, i == 1 ? 0 : 1, q, j, k)];
    return lat_load(L, g, q, i, j, k);
}

// Value a later lattice load returns for an arithmetic value v of population q.
template <typename S, typename R>
__device__ __forceinline__ R stored_value(R v, int q, R scale, R inv_scale) {
    return Store<S, R>::load(Store<S, R>::store(v, q, scale), q, inv_scale);
}
template <typename S, typename R>
__device__ __forceinline__ void ghost_store(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k, R v) {
    L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)] = v;
}

// ---------------------------------------------------------------------------
// BGK collision of one node, CODE/SRC/col.F90:127-229, same operation order.
// x[0..17] are the streamed populations b01..b18, x[18] is a19; on return x
// holds a01..a19 after collision.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void collide(R* x, R omega, R omega1, R fgrad) {
    const R uno = R(1), tre = R(3), qf = R(1.5), rf = R(3), zero = R(0);
    const R p0 = Const<R>::p0(), p1 = Const<R>::p1(), p2 = Const<R>::p2();
    const R drho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7] + x[8] + x[9] + x[10] +
                   x[11] + x[12] + x[13] + x[14] + x[15] + x[16] + x[17] + x[18];
    const R drhoinv = uno / drho;
    R dvx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * drhoinv;
    R dvy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * drhoinv;
    R dvz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * drhoinv;
    const R dvx2 = dvx * dvx, dvy2 = dvy * dvy, dvz2 = dvz * dvz;
    const R dvsq = dvx2 + dvy2 + dvz2;
    R dvxpy = dvx + dvy;
    const R dqxpy = uno + qf * (tre * dvxpy * dvxpy - dvsq);
    R dvxmy = dvx - dvy;
    const R dqxmy = uno + qf * (tre * dvxmy * dvxmy - dvsq);
    R dvxpz = dvx + dvz;
    const R dqxpz = uno + qf * (tre * dvxpz * dvxpz - dvsq);
    R dvxmz = dvx - dvz;
    const R dqxmz = uno + qf * (tre * dvxmz * dvxmz - dvsq);
    R dvypz = dvy + dvz;
    const R dqypz = uno + qf * (tre * dvypz * dvypz - dvsq);
    R dvymz = dvy - dvz;
    const R dqymz = uno + qf * (tre * dvymz * dvymz - dvsq);
    const R dqx = uno + qf * (tre * dvx2 - dvsq);
    const R dqy = uno + qf * (tre * dvy2 - dvsq);
    const R dqz = uno + qf * (tre * dvz2 - dvsq);
    dvx = rf * dvx; dvy = rf * dvy; dvz = rf * dvz;
    dvxpy = rf * dvxpy; dvxmy = rf * dvxmy; dvxpz = rf * dvxpz;
    dvxmz = rf * dvxmz; dvypz = rf * dvypz; dvymz = rf * dvymz;
    const R drp1 = drho * p1;
    const R drp2 = drho * p2;
    const R forcex = fgrad * drho, forcey = zero, forcez = zero;  // FORCING_X (default)

    const R de01 = drp2 * (dvxmy + dqxmy);
    const R de02 = drp2 * (dvxmz + dqxmz);
    const R de03 = drp2 * (dvxpy + dqxpy);
    const R de04 = drp2 * (dvxpz + dqxpz);
    const R de05 = drp1 * (dvx + dqx);
    const R de06 = drp1 * (dvz + dqz);
    const R de07 = drp2 * (dvypz + dqypz);
    const R de08 = drp1 * (dvy + dqy);
    const R de09 = drp2 * (dvymz + dqymz);
    const R de10 = drp2 * (-dvxpy + dqxpy);
    const R de11 = drp2 * (-dvxpz + dqxpz);
    const R de12 = drp2 * (-dvxmy + dqxmy);
    const R de13 = drp2 * (-dvxmz + dqxmz);
    const R de14 = drp1 * (-dvx + dqx);
    const R de15 = drp1 * (-dvz + dqz);
    const R de16 = drp2 * (-dvypz + dqypz);
    const R de17 = drp1 * (-dvy + dqy);
    const R de18 = drp2 * (-dvymz + dqymz);
    const R de19 = drho * p0 * (uno - qf * dvsq);

    x[0] = omega1 * x[0] + (omega * de01 + forcex - forcey);
    x[1] = omega1 * x[1] + (omega * de02 + forcex - forcez);
    x[2] = omega1 * x[2] + (omega * de03 + forcex + forcey);
    x[3] = omega1 * x[3] + (omega * de04 + forcex + forcez);
    x[4] = omega1 * x[4] + (omega * de05 + forcex);
    x[5] = omega1 * x[5] + (omega * de06 + forcez);
    x[6] = omega1 * x[6] + (omega * de07 + forcey + forcez);
    x[7] = omega1 * x[7] + (omega * de08 + forcey);
    x[8] = omega1 * x[8] + (omega * de09 + forcey - forcez);
    x[9] = omega1 * x[9] + (omega * de10 - forcex - forcey);
    x[10] = omega1 * x[10] + (omega * de11 - forcex - forcez);
    x[11] = omega1 * x[11] + (omega * de12 - forcex + forcey);
    x[12] = omega1 * x[12] + (omega * de13 - forcex + forcez);
    x[13] = omega1 * x[13] + (omega * de14 - forcex);
    x[14] = omega1 * x[14] + (omega * de15 - forcez);
    x[15] = omega1 * x[15] + (omega * de16 - forcey - forcez);
    x[16] = omega1 * x[16] + (omega * de17 - forcey);
    x[17] = omega1 * x[17] + (omega * de18 - forcey + forcez);
    x[18] = omega1 * x[18] + (omega * de19);
}

// ---------------------------------------------------------------------------
// 16-bit storage works on the stored quantity itself, D_q = (f_q - w_q)*S.
// Because sum_q w_q = 1 and sum_q w_q c_q = 0, density and momentum follow
// from D directly (rho - 1 = sum D / S, j = sum c D / S), and BGK maps
// deviations to deviations:
//   D'_q = (1-omega) D_q + S [omega (feq_q - w_q) + F_q],
//   feq_q - w_q = w_q [(rho-1) + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u^2)],
// the equilibrium of CODE/SRC/col.F90:190-208 written about w_q.  Loads and
// stores are then plain conversions and no step subtracts two nearly equal
// numbers.  Arithmetic is FP32 with explicit fused multiply-adds.
// ---------------------------------------------------------------------------
template <typename S> struct DevStore { static constexpr bool value = false; };
template <> struct DevStore<__half> {
    static constexpr bool value = true;
    static __device__ __forceinline__ float to_f(__half s) { return __half2float(s); }
    static __device__ __forceinline__ __half from_f(float d) { return __float2half_rn(d); }
    static __device__ __forceinline__ __half from_d(double d) { return __double2half(d); }
};
template <> struct DevStore<__nv_bfloat16> {
    static constexpr bool value = true;
    static __device__ __forceinline__ float to_f(__nv_bfloat16 s) { return __bfloat162float(s); }
    static __device__ __forceinline__ __nv_bfloat16 from_f(float d) { return __float2bfloat16_rn(d); }
    static __device__ __forceinline__ __nv_bfloat16 from_d(double d) { return __double2bfloat16(d); }
};

// Reciprocal for the 16-bit path: the hardware approximation (rcp.approx, relative
// error below 2^-22), per lane, so the one-node and two-node kernels agree bit for bit.
__device__ __forceinline__ float rcp_dev(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ F2 rcp_dev(F2 x) { return F2(rcp_dev(x.v.x), rcp_dev(x.v.y)); }

// One opposite pair (qp, qm) with c_qp . u = v, c_qm = -c_qp; FX = +-1/0 the x
// component of c_qp (the body force acts along x).  With c0 = (rho-1) - 1.5 rho u^2,
//   D'_qp = (1-omega) D_qp + S omega w [c0 + 4.5 rho v^2 + 3 rho v] + S F_qp
// and D'_qm the same with -v.  V = float, or F2 for two nodes.
template <int FX, typename V>
__device__ __forceinline__ void dev_pair(V* D, int qp, int qm, V v, V ow, V c0, V r45, V r3, float omega1, V fS) {
    const V a = fma_rn(r45 * v, v, c0);
    const V b = r3 * v;
    const V dp = FX != 0 ? fma_rn(V(omega1), D[qp], fS) : V(omega1) * D[qp];
    const V dm = FX != 0 ? fma_rn(V(omega1), D[qm], -fS) : V(omega1) * D[qm];
    D[qp] = fma_rn(ow, a + b, dp);
    D[qm] = fma_rn(ow, a - b, dm);
}

template <typename V>
__device__ __forceinline__ void collide_dev(V* D, float omega, float omega1, float fgrad, float S, float invS) {
    // rho - 1 and j from partial sums shared between the moments: the +x and -x groups,
    // the y+ and y- populations without an x component, and the rest
    const V xp = ((D[0] + D[1]) + (D[2] + D[3])) + D[4];
    const V xm = ((D[9] + D[10]) + (D[11] + D[12])) + D[13];
    const V yp = (D[6] + D[7]) + D[8];
    const V ym = (D[15] + D[16]) + D[17];
    const V z0 = (D[5] + D[14]) + D[18];
    const V s = ((xp + xm) + (yp + ym)) + z0;
    const V jx = xp - xm;
    const V jy = ((D[2] + D[11]) + yp) - ((D[0] + D[9]) + ym);
    const V jz = ((D[3] + D[5]) + (D[6] + D[12]) + D[17]) - ((D[1] + D[8]) + (D[10] + D[14]) + D[15]);
    const V rm1 = s * V(invS);
    const V rho = V(1.0f) + rm1;
    const V ri = V(invS) * rcp_dev(rho);
    const V ux = jx * ri, uy = jy * ri, uz = jz * ri;
    const V r15 = V(1.5f) * rho;
    const V c0 = fma_rn(-r15, fma_rn(ux, ux, fma_rn(uy, uy, uz * uz)), rm1);  // (rho-1) - 1.5 rho u^2
    const V r45 = V(4.5f) * rho, r3 = V(3.0f) * rho;
    const V fS = V(S * fgrad) * rho;
    const float oS = omega * S;
    const V ow1 = V(oS * (1.0f / 18.0f)), ow2 = V(oS * (1.0f / 36.0f)), ow0 = V(oS * (1.0f / 3.0f));
    dev_pair<1>(D, 4, 13, ux, ow1, c0, r45, r3, omega1, fS);        // a05 / a14
    dev_pair<0>(D, 5, 14, uz, ow1, c0, r45, r3, omega1, fS);        // a06 / a15
    dev_pair<0>(D, 7, 16, uy, ow1, c0, r45, r3, omega1, fS);        // a08 / a17
    dev_pair<1>(D, 0, 11, ux - uy, ow2, c0, r45, r3, omega1, fS);   // a01 / a12
    dev_pair<1>(D, 1, 12, ux - uz, ow2, c0, r45, r3, omega1, fS);   // a02 / a13
    dev_pair<1>(D, 2, 9, ux + uy, ow2, c0, r45, r3, omega1, fS);    // a03 / a10
    dev_pair<1>(D, 3, 10, ux + uz, ow2, c0, r45, r3, omega1, fS);   // a04 / a11
    dev_pair<0>(D, 6, 15, uy + uz, ow2, c0, r45, r3, omega1, fS);   // a07 / a16
    dev_pair<0>(D, 8, 17, uy - uz, ow2, c0, r45, r3, omega1, fS);   // a09 / a18
    D[18] = fma_rn(ow0, c0, V(omega1) * D[18]);                      // a19
}

// Physical constants of one run, rounded to the arithmetic type the way
// CODE/SRC/hencol.F90:30-39 rounds them to mykind.
template <typename R>
struct Phys {
    R omega, omega1, fgrad, u_inflow, force;
};

}  // namespace eup

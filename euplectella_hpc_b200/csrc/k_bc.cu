// Boundary side of the time step: halo planes (CODE/SRC/bcond.bc.F90),
// bounce-back on solid voxels with the momentum-exchange force
// (CODE/SRC/bcond.obs.F90), the FP64 monitor (CODE/SRC/diagno.F90), probes
// (CODE/SRC/probe_global.F90) and the host-layout scatter/gather used by
// upload and download.  All of it is O(surface) or O(solid surface) work.
#include "init_eq.h"
#include <algorithm>
#include <type_traits>

#include "internal.h"

namespace eup {

namespace {

// One thread per (a, b) pair of a face loop; a runs fastest.
struct Range2 {
    int a0, na, b0, nb;
    // element `t` of the loop (false beyond its end)
    __device__ __forceinline__ bool at(int64_t t, int& a, int& b) const {
        if (t >= (int64_t)na * nb) return false;
        a = a0 + (int)(t % na);
        b = b0 + (int)(t / na);
        return true;
    }
    int64_t size() const { return (int64_t)na * nb; }
    unsigned blocks(int tpb) const {
        const int64_t t = (int64_t)na * nb;
        return (unsigned)((t + tpb - 1) / tpb);
    }
};

constexpr int kTpb = 256;

// Loads inside the halo kernels go through bc_load: interior nodes of the
// x = 1 and x = l columns come from the compact x-face copy written by the
// stream-collide kernel (coalesced in j), other interior nodes from the
// lattice, halo nodes from the shell.  Every kernel issues all of a thread's
// loads before its first store (stores to the shell may alias the loads).
#define LD(q1, i, j, k) bc_load(L, g, (q1) - 1, (i), (j), (k))
#define ST(q1, i, j, k, v) ghost_store(L, g, (q1) - 1, (i), (j), (k), (v))

// ---- front wall, x = l+1 -----------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void front_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, int64_t tid) {
    int j, k;
    if (!r.at(tid, j, k)) return;
    const int l = g.l, l1 = g.l + 1, m = g.m;
    if (flag == 0) {  // periodic, CODE/SRC/bcond.bc.F90:75-105 (SERIAL corner line :90)
        if (j == 0) { const R v = LD(12, 1, m, k); ST(12, l1, 0, k, v); return; }
        R v[5];
#pragma unroll
        for (int q = 10; q <= 14; ++q) v[q - 10] = LD(q, 1, j, k);
#pragma unroll
        for (int q = 10; q <= 14; ++q) ST(q, l1, j, k, v[q - 10]);
    } else if (flag == 1) {  // no-slip, :108-124
        const R v1 = LD(1, l, j, k), v2 = LD(2, l, j, k), v3 = LD(3, l, j, k), v4 = LD(4, l, j, k), v5 = LD(5, l, j, k);
        ST(12, l1, j - 1, k, v1);
        ST(13, l1, j, k - 1, v2);
        ST(10, l1, j + 1, k, v3);
        ST(11, l1, j, k + 1, v4);
        ST(14, l1, j, k, v5);
    } else {  // outflow, :127-169: equilibrium at rho=1 with the (un-normalised) momentum of x=l
        R a[18];
#pragma unroll
        for (int q = 0; q < 18; ++q) a[q] = bc_load(L, g, q, l, j, k);
        const R xj = a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13];
        const R yj = a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17];
        const R zj = a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15];
        const R rf = R(3), qf = R(1.5), t3 = R(3), one = R(1);
        const R cvsq = xj * xj + yj * yj + zj * zj;
        const R cx10 = rf * (-xj - yj) + qf * (t3 * (xj + yj) * (xj + yj) - cvsq);
        const R cx11 = rf * (-xj - zj) + qf * (t3 * (xj + zj) * (xj + zj) - cvsq);
        const R cx12 = rf * (-xj + yj) + qf * (t3 * (xj - yj) * (xj - yj) - cvsq);
        const R cx13 = rf * (-xj + zj) + qf * (t3 * (xj - zj) * (xj - zj) - cvsq);
        const R cx14 = rf * (-xj) + qf * (t3 * (xj) * (xj) - cvsq);
        const R p1 = Const<R>::p1(), p2 = Const<R>::p2();
        ST(10, l1, j, k, p2 * (one + cx10));
        ST(11, l1, j, k, p2 * (one + cx11));
        ST(12, l1, j, k, p2 * (one + cx12));
        ST(13, l1, j, k, p2 * (one + cx13));
        ST(14, l1, j, k, p1 * (one + cx14));
    }
}

// Outflow border fix, CODE/SRC/bcond.bc.F90:172-203: copies of the edge rows.
template <typename S, typename R>
__device__ __forceinline__ void front_fix_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int64_t tid) {
    int t, side;
    if (!r.at(tid, t, side)) return;
    const int l1 = g.l + 1, m = g.m, n = g.n;
    R lo[5], hi[5];
    if (side == 0 && t >= 1 && t <= m) {
#pragma unroll
        for (int q = 10; q <= 14; ++q) { lo[q - 10] = LD(q, l1, t, 1); hi[q - 10] = LD(q, l1, t, n); }
#pragma unroll
        for (int q = 10; q <= 14; ++q) { ST(q, l1, t, 0, lo[q - 10]); ST(q, l1, t, n + 1, hi[q - 10]); }
    }
    if (side == 1 && t >= 1 && t <= n) {
#pragma unroll
        for (int q = 10; q <= 14; ++q) { lo[q - 10] = LD(q, l1, 1, t); hi[q - 10] = LD(q, l1, m, t); }
#pragma unroll
        for (int q = 10; q <= 14; ++q) { ST(q, l1, 0, t, lo[q - 10]); ST(q, l1, m + 1, t, hi[q - 10]); }
    }
}

// ---- rear wall, x = 0 ----------------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void rear_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, R u_inflow, int64_t tid) {
    int j, k;
    if (!r.at(tid, j, k)) return;
    const int l = g.l, m1 = g.m + 1;
    if (flag == 0) {  // periodic, :210-238 (SERIAL corner line :223)
        if (j == 0) { const R v = LD(1, l, 1, k); ST(1, 0, m1, k, v); return; }
        R v[5];
#pragma unroll
        for (int q = 1; q <= 5; ++q) v[q - 1] = LD(q, l, j, k);
#pragma unroll
        for (int q = 1; q <= 5; ++q) ST(q, 0, j, k, v[q - 1]);
    } else if (flag == 1) {  // no-slip, :241-257
        const R v10 = LD(10, 1, j, k), v11 = LD(11, 1, j, k), v12 = LD(12, 1, j, k), v13 = LD(13, 1, j, k),
                v14 = LD(14, 1, j, k);
        ST(3, 0, j - 1, k, v10);
        ST(4, 0, j, k - 1, v11);
        ST(1, 0, j + 1, k, v12);
        ST(2, 0, j, k + 1, v13);
        ST(5, 0, j, k, v14);
    } else {  // inflow, uniform, :260-321
        const R xj = u_inflow, yj = R(0), zj = R(0);
        const R rf = R(3), qf = R(1.5), t3 = R(3), one = R(1);
        const R cvsq = xj * xj + yj * yj + zj * zj;
        const R cx01 = rf * (xj - yj) + qf * (t3 * (xj - yj) * (xj - yj) - cvsq);
        const R cx02 = rf * (xj - zj) + qf * (t3 * (xj - zj) * (xj - zj) - cvsq);
        const R cx03 = rf * (xj + yj) + qf * (t3 * (xj + yj) * (xj + yj) - cvsq);
        const R cx04 = rf * (xj + zj) + qf * (t3 * (xj + zj) * (xj + zj) - cvsq);
        const R cx05 = rf * (xj) + qf * (t3 * (xj) * (xj) - cvsq);
        const R p1 = Const<R>::p1(), p2 = Const<R>::p2();
        ST(1, 0, j, k, p2 * (one + cx01));
        ST(2, 0, j, k, p2 * (one + cx02));
        ST(3, 0, j, k, p2 * (one + cx03));
        ST(4, 0, j, k, p2 * (one + cx04));
        ST(5, 0, j, k, p1 * (one + cx05));
    }
}

// ---- up wall, z = n+1 -------------------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void up_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, R force, int64_t tid) {
    int i, j;
    if (!r.at(tid, i, j)) return;
    const int n = g.n, n1 = g.n + 1;
    if (flag == 0) {  // periodic, :385-409
        const R v2 = LD(2, i, j, 1), v9 = LD(9, i, j, 1), v11 = LD(11, i, j, 1), v15 = LD(15, i, j, 1),
                v16 = LD(16, i, j, 1);
        ST(2, i, j, n1, v2);
        ST(9, i, j, n1, v9);
        ST(11, i, j, n1, v11);
        ST(15, i, j, n1, v15);
        ST(16, i, j, n1, v16);
    } else if (flag == 1 || flag == 2) {  // no-slip :412-428, lid :431-447
        const R v6 = LD(6, i, j, n), v13 = LD(13, i, j, n), v18 = LD(18, i, j, n), v4 = LD(4, i, j, n),
                v7 = LD(7, i, j, n);
        ST(15, i, j, n1, v6);
        ST(2, i - 1, j, n1, flag == 2 ? v13 + force : v13);
        ST(9, i, j - 1, n1, v18);
        ST(11, i + 1, j, n1, flag == 2 ? v4 - force : v4);
        ST(16, i, j + 1, n1, v7);
    } else {  // free-slip over i = 0..l+1, j = 0..m+1, :450-468
        const R v6 = LD(6, i, j, n), v13 = LD(13, i, j, n), v18 = LD(18, i, j, n), v4 = LD(4, i, j, n),
                v7 = LD(7, i, j, n);
        ST(15, i, j, n1, v6);
        ST(11, i, j, n1, v13);
        ST(16, i, j, n1, v18);
        ST(2, i, j, n1, v4);
        ST(9, i, j, n1, v7);
    }
}

// ---- down wall, z = 0 ---------------------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void down_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, int64_t tid) {
    int i, j;
    if (!r.at(tid, i, j)) return;
    const int n = g.n;
    if (flag == 0) {  // periodic, :472-496
        const R v4 = LD(4, i, j, n), v6 = LD(6, i, j, n), v7 = LD(7, i, j, n), v13 = LD(13, i, j, n),
                v18 = LD(18, i, j, n);
        ST(4, i, j, 0, v4);
        ST(6, i, j, 0, v6);
        ST(7, i, j, 0, v7);
        ST(13, i, j, 0, v13);
        ST(18, i, j, 0, v18);
    } else if (flag == 1) {  // no-slip, :499-515
        const R v15 = LD(15, i, j, 1), v11 = LD(11, i, j, 1), v16 = LD(16, i, j, 1), v2 = LD(2, i, j, 1),
                v9 = LD(9, i, j, 1);
        ST(6, i, j, 0, v15);
        ST(4, i - 1, j, 0, v11);
        ST(7, i, j - 1, 0, v16);
        ST(13, i + 1, j, 0, v2);
        ST(18, i, j + 1, 0, v9);
    } else {  // free-slip, :518-530
        const R v15 = LD(15, i, j, 1), v11 = LD(11, i, j, 1), v16 = LD(16, i, j, 1), v2 = LD(2, i, j, 1),
                v9 = LD(9, i, j, 1);
        ST(6, i, j, 0, v15);
        ST(13, i, j, 0, v11);
        ST(18, i, j, 0, v16);
        ST(4, i, j, 0, v2);
        ST(7, i, j, 0, v9);
    }
}

// ---- left wall, y = 0 ------------------------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void left_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, int64_t tid) {
    int i, k;
    if (!r.at(tid, i, k)) return;
    const int l = g.l, m = g.m;
    if (flag == 0) {  // periodic, :535-560 (corner line :547)
        if (i == 0) { const R v = LD(3, l, m, k); ST(3, 0, 0, k, v); return; }
        const R v3 = LD(3, i, m, k), v7 = LD(7, i, m, k), v8 = LD(8, i, m, k), v9 = LD(9, i, m, k),
                v12 = LD(12, i, m, k);
        ST(3, i, 0, k, v3);
        ST(7, i, 0, k, v7);
        ST(8, i, 0, k, v8);
        ST(9, i, 0, k, v9);
        ST(12, i, 0, k, v12);
    } else if (flag == 1) {  // no-slip, :563-579
        const R v17 = LD(17, i, 1, k), v1 = LD(1, i, 1, k), v10 = LD(10, i, 1, k), v16 = LD(16, i, 1, k),
                v18 = LD(18, i, 1, k);
        ST(8, i, 0, k, v17);
        ST(12, i + 1, 0, k, v1);
        ST(3, i - 1, 0, k, v10);
        ST(7, i, 0, k - 1, v16);
        ST(9, i, 0, k + 1, v18);
    } else {  // free-slip, :582-594
        const R v17 = LD(17, i, 1, k), v1 = LD(1, i, 1, k), v10 = LD(10, i, 1, k), v16 = LD(16, i, 1, k),
                v18 = LD(18, i, 1, k);
        ST(8, i, 0, k, v17);
        ST(3, i, 0, k, v1);
        ST(12, i, 0, k, v10);
        ST(9, i, 0, k, v16);
        ST(7, i, 0, k, v18);
    }
}

// ---- right wall, y = m+1 ------------------------------------------------------------------
template <typename S, typename R>
__device__ __forceinline__ void right_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int flag, int64_t tid) {
    int i, k;
    if (!r.at(tid, i, k)) return;
    const int m = g.m, m1 = g.m + 1, l1 = g.l + 1;
    if (flag == 0) {  // periodic, :600-625 (corner line :612)
        if (i == 0) { const R v = LD(10, 1, 1, k); ST(10, l1, m1, k, v); return; }
        const R v1 = LD(1, i, 1, k), v10 = LD(10, i, 1, k), v16 = LD(16, i, 1, k), v17 = LD(17, i, 1, k),
                v18 = LD(18, i, 1, k);
        ST(1, i, m1, k, v1);
        ST(10, i, m1, k, v10);
        ST(16, i, m1, k, v16);
        ST(17, i, m1, k, v17);
        ST(18, i, m1, k, v18);
    } else if (flag == 1) {  // no-slip, :628-644
        const R v3 = LD(3, i, m, k), v7 = LD(7, i, m, k), v8 = LD(8, i, m, k), v9 = LD(9, i, m, k),
                v12 = LD(12, i, m, k);
        ST(10, i + 1, m1, k, v3);
        ST(16, i, m1, k + 1, v7);
        ST(17, i, m1, k, v8);
        ST(18, i, m1, k - 1, v9);
        ST(1, i - 1, m1, k, v12);
    } else {  // free-slip, :647-659
        const R v3 = LD(3, i, m, k), v7 = LD(7, i, m, k), v8 = LD(8, i, m, k), v9 = LD(9, i, m, k),
                v12 = LD(12, i, m, k);
        ST(1, i, m1, k, v3);
        ST(18, i, m1, k, v7);
        ST(17, i, m1, k, v8);
        ST(16, i, m1, k, v9);
        ST(10, i, m1, k, v12);
    }
}

// Free-slip edge fixes, CODE/SRC/bcond.bc.F90:663-690.
template <typename S, typename R>
__device__ __forceinline__ void edge_fix_body(const Lat<S, R>& L, const Geo& g, const Range2& r, int fixes, int64_t tid) {
    int i, dummy;
    if (!r.at(tid, i, dummy)) return;
    const int m = g.m, m1 = g.m + 1, n = g.n, n1 = g.n + 1;
    const R v1 = (fixes & 1) ? LD(18, i, 1, n) : R(0);
    const R v2 = (fixes & 2) ? LD(7, i, m, n) : R(0);
    const R v3 = (fixes & 4) ? LD(9, i, m, 1) : R(0);
    const R v4 = (fixes & 8) ? LD(16, i, 1, 1) : R(0);
    if (fixes & 1) ST(9, i, 0, n1, v1);
    if (fixes & 2) ST(16, i, m1, n1, v2);
    if (fixes & 4) ST(18, i, m1, 0, v3);
    if (fixes & 8) ST(7, i, 0, 0, v4);
}

#undef LD
#undef ST

// ---- bounce-back + momentum exchange ---------------------------------------------------
//
// For each solid voxel x touching fluid or halo and each moving q, the
// reference sets a_q(x) = a_opp(q)(x + c_q) (CODE/SRC/bcond.obs.F90:56-73), so
// that the next pull returns to the fluid node x + c_q its own post-collision
// population.  Links whose neighbour is itself solid are skipped: their value
// is only ever pulled into solid voxels.  The same reads give the force: the
// population a_opp(q)(y) leaving fluid node y = x + c_q towards x transfers
// 2 c_opp(q) a_opp(q)(y) = -2 c_q a_opp(q)(y); across a periodic axis y is the
// wrapped node and its interior value is used.  The force of the state read
// goes to series[itime % cap], itime read from device memory; with `advance`
// the last block then increments the device step counter.

// One kernel per halo block (the reference's blocks as separate launches).
template <typename S, typename R>
__global__ void k_front(Lat<S, R> L, Geo g, Range2 r, int flag) {
    front_body<S, R>(L, g, r, flag, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_front_fix(Lat<S, R> L, Geo g, Range2 r) {
    front_fix_body<S, R>(L, g, r, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_rear(Lat<S, R> L, Geo g, Range2 r, int flag, R u_inflow) {
    rear_body<S, R>(L, g, r, flag, u_inflow, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_up(Lat<S, R> L, Geo g, Range2 r, int flag, R force) {
    up_body<S, R>(L, g, r, flag, force, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_down(Lat<S, R> L, Geo g, Range2 r, int flag) {
    down_body<S, R>(L, g, r, flag, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_left(Lat<S, R> L, Geo g, Range2 r, int flag) {
    left_body<S, R>(L, g, r, flag, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_right(Lat<S, R> L, Geo g, Range2 r, int flag) {
    right_body<S, R>(L, g, r, flag, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename S, typename R>
__global__ void k_edge_fix(Lat<S, R> L, Geo g, Range2 r, int fixes) {
    edge_fix_body<S, R>(L, g, r, fixes, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---- all halo blocks in one launch (opt-in: EUP_STEP_VARIANT bit 12) ------------------
// Measured slower than one launch per block on B200 (768x384x384: 0.100 ms against 0.060 ms
// of halo planes per step; 192x96x96 as well), kept as a tested alternative.
// The blocks of one step as phases of a single kernel, in the same order, with a grid-wide
// barrier between phases where the separate launches had a kernel boundary: every element of
// a phase sees every store of the phases before it, exactly as with one launch per block, so
// the results are the same bits.  The grid is launched cooperatively (all CTAs resident); the
// barrier is this library's own (one arrival counter and one generation word per handle, in
// device memory), and its wait is bounded: after kBarrierWaitNs it counts a timeout in the
// barrier's third word, which the host reports, and goes on instead of waiting forever.
enum : int { kBcFront = 0, kBcFrontFix, kBcRear, kBcUp, kBcDown, kBcLeft, kBcRight, kBcEdgeFix };
struct BcPhase {
    int kind, flag;
    Range2 r;
};
template <typename R>
struct BcPlan {
    int n;
    BcPhase ph[8];
    R u_inflow, force;
};

constexpr uint64_t kBarrierWaitNs = 1000000000ull;

__device__ __forceinline__ uint64_t bc_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bar[0] arrivals, bar[1] generation, bar[2] timeouts (zero when the handle is created)
__device__ __forceinline__ void grid_barrier(unsigned int* bar) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = bar + 1;
        const unsigned int g0 = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(bar, 1u) + 1u;
        if (arrived == gridDim.x) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const uint64_t t0 = bc_ns();
            while (*gen == g0) {
                if (bc_ns() - t0 > kBarrierWaitNs) {
                    atomicAdd(bar + 2, 1u);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <typename S, typename R>
__global__ void __launch_bounds__(kTpb) k_bc_all(Lat<S, R> L, Geo g, BcPlan<R> plan, unsigned int* bar) {
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    for (int p = 0; p < plan.n; ++p) {
        const BcPhase ph = plan.ph[p];
        const int64_t work = (int64_t)ph.r.na * ph.r.nb;
        for (int64_t t = t0; t < work; t += nt) {
            switch (ph.kind) {
                case kBcFront: front_body<S, R>(L, g, ph.r, ph.flag, t); break;
                case kBcFrontFix: front_fix_body<S, R>(L, g, ph.r, t); break;
                case kBcRear: rear_body<S, R>(L, g, ph.r, ph.flag, plan.u_inflow, t); break;
                case kBcUp: up_body<S, R>(L, g, ph.r, ph.flag, plan.force, t); break;
                case kBcDown: down_body<S, R>(L, g, ph.r, ph.flag, t); break;
                case kBcLeft: left_body<S, R>(L, g, ph.r, ph.flag, t); break;
                case kBcRight: right_body<S, R>(L, g, ph.r, ph.flag, t); break;
                default: edge_fix_body<S, R>(L, g, ph.r, ph.flag, t); break;
            }
        }
        if (p + 1 < plan.n) grid_barrier(bar);
    }
}

// Co-resident CTAs of k_bc_all per device and storage type (0: not measured / not usable).
constexpr int kBcMaxDevices = 64;
int g_bc_fused_blocks[kBcMaxDevices][4] = {};
bool g_bc_fused_ok[kBcMaxDevices] = {};

template <typename S> constexpr int bc_type_index() {
    return sizeof(S) == 4 ? 0 : sizeof(S) == 8 ? 1 : std::is_same<S, __half>::value ? 2 : 3;
}

__global__ void k_coop_probe(unsigned int* bar) { grid_barrier(bar); }

template <typename S, typename R>
__global__ void k_bounce_drag(Lat<S, R> L, Geo g, int per_x, int per_y, int per_z, const int32_t* list,
                              const uint64_t* links, int64_t nlist, int do_bounce, Reduce red, double* series,
                              int64_t cap, int64_t* d_itime, int advance) {
    double f[3] = {0.0, 0.0, 0.0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nlist;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t lin = list[t];
        const uint64_t w = links[t];
        const uint32_t fl = (uint32_t)(w & 0x3FFFFu);          // neighbour x + c_q is interior fluid
        const uint32_t gh = (uint32_t)((w >> 18) & 0x3FFFFu);  // neighbour is a halo node
        const uint32_t wf = (uint32_t)((w >> 36) & 0x3FFFFu);  // halo neighbour wraps onto interior fluid
        const int i = lin % g.l + 1;
        const int jk = lin / g.l;
        const int j = jk % g.m + 1, k = jk / g.m + 1;
        S raw[18];
        R val[18];
        // all loads first: interior fluid neighbours from the lattice, halo ones from the shell
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const int qo = opp_of(q);
            raw[q] = S();
            if ((fl >> q) & 1u) {
                raw[q] = L.pop[qo][(int64_t)lin + cx_of(q) + (int64_t)cy_of(q) * g.l + (int64_t)cz_of(q) * g.lm];
            } else if ((gh >> q) & 1u) {
                const R v = L.ghost[(int64_t)qo * g.G + g.gidx(i + cx_of(q), j + cy_of(q), k + cz_of(q))];
                raw[q] = Store<S, R>::store(v, q, L.scale);
            }
        }
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            val[q] = ((fl >> q) & 1u) ? Store<S, R>::load(raw[q], opp_of(q), L.inv_scale)
                                      : Store<S, R>::load(raw[q], q, L.inv_scale);
            if ((fl >> q) & 1u) {
                const double v = (double)val[q];
                f[0] -= 2.0 * cx_of(q) * v;
                f[1] -= 2.0 * cy_of(q) * v;
                f[2] -= 2.0 * cz_of(q) * v;
            }
        }
        if (wf) {  // links across a periodic axis: force from the wrapped fluid node
#pragma unroll
            for (int q = 0; q < 18; ++q) {
                if (!((wf >> q) & 1u)) continue;
                int wi = i + cx_of(q), wj = j + cy_of(q), wk = k + cz_of(q);
                if (per_x) wi = wi < 1 ? wi + g.l : (wi > g.l ? wi - g.l : wi);
                if (per_y) wj = wj < 1 ? wj + g.m : (wj > g.m ? wj - g.m : wj);
                if (per_z) wk = wk < 1 ? wk + g.n : (wk > g.n ? wk - g.n : wk);
                const double v = (double)lat_load(L, g, opp_of(q), wi, wj, wk);
                f[0] -= 2.0 * cx_of(q) * v;
                f[1] -= 2.0 * cy_of(q) * v;
                f[2] -= 2.0 * cz_of(q) * v;
            }
        }
        if (do_bounce) {
            const uint32_t wr = fl | gh;
#pragma unroll
            for (int q = 0; q < 18; ++q)
                if ((wr >> q) & 1u) L.pop[q][lin] = raw[q];
            if (i == 1 || i == g.l) {
#pragma unroll
                for (int q = 0; q < 18; ++q) {
                    if (!((wr >> q) & 1u)) continue;
                    if (i == 1) L.xface[xface_idx(g, 0, q, j, k)] = val[q];
                    if (i == g.l) L.xface[xface_idx(g, 1, q, j, k)] = val[q];
                }
            }
        }
    }
    block_reduce_store<3>(f, red, nullptr, series, cap, d_itime, advance);
}

// ---- FP64 monitor, CODE/SRC/diagno.F90:67-120 -------------------------------------------
template <typename S, typename R>
__global__ void k_monitor(Lat<S, R> L, Geo g, Mask mk, Reduce red, double* out) {
    double s[5] = {0, 0, 0, 0, 0};
    for (int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.N;
         lin += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(lin % g.l) + 1;
        const int j = (int)((lin / g.l) % g.m) + 1;
        const int k = (int)(lin / g.lm) + 1;
        if (mk.solid(g, i, j, k)) {
            s[0] += 1.0;
            continue;
        }
        double a[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) a[q] = (double)Store<S, R>::load(L.pop[q][lin], q, L.inv_scale);
        double rho = 0.0;
#pragma unroll
        for (int q = 0; q < 19; ++q) rho += a[q];
        const double ri = 1.0 / rho;
        const double xj = (a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13]) * ri;
        const double yj = (a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17]) * ri;
        const double zj = (a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15]) * ri;
        s[0] += rho; s[1] += xj; s[2] += yj; s[3] += zj; s[4] += xj * xj + yj * yj + zj * zj;
    }
    block_reduce_store<5>(s, red, out);
}

// FP64 sums over the fluid nodes with region[lin] != 0 (the cavity of a shell,
// a probe box, ...): {count, sum rho, sum ux, sum uy, sum uz, sum u^2}, u = j/rho
// as CODE/SRC/diagno.F90:86-105 computes it.
template <typename S, typename R>
__global__ void k_region_sums(Lat<S, R> L, Geo g, Mask mk, const uint8_t* region, Reduce red, double* out) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.N;
         lin += (int64_t)gridDim.x * blockDim.x) {
        if (!region[lin]) continue;
        const int i = (int)(lin % g.l) + 1;
        const int j = (int)((lin / g.l) % g.m) + 1;
        const int k = (int)(lin / g.lm) + 1;
        if (mk.solid(g, i, j, k)) continue;
        double a[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) a[q] = (double)Store<S, R>::load(L.pop[q][lin], q, L.inv_scale);
        double rho = 0.0;
#pragma unroll
        for (int q = 0; q < 19; ++q) rho += a[q];
        const double ri = 1.0 / rho;
        const double xj = (a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13]) * ri;
        const double yj = (a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17]) * ri;
        const double zj = (a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15]) * ri;
        s[0] += 1.0; s[1] += rho; s[2] += xj; s[3] += yj; s[4] += zj; s[5] += xj * xj + yj * yj + zj * zj;
    }
    block_reduce_store<6>(s, red, out);
}

// ---- reference-form diagnostics: line profiles, plane means, control-volume drag ----------

// Macroscopic values of one interior node in R, in the expression order of
// CODE/SRC/prof_i.F90:45-79 (div = true: momentum / den) and
// CODE/SRC/varm.F90:53-85 (div = false: momentum * (1 / den)).
template <typename S, typename R>
__device__ __forceinline__ void ref_macro(const Lat<S, R>& L, int64_t lin, bool div, R& den, R& u, R& w, R& v) {
    R f[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = Store<S, R>::load(L.pop[q][lin], q, L.inv_scale);
    const R r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] +
                f[14] + f[15] + f[16] + f[17] + f[18];
    const R mx = f[0] + f[1] + f[2] + f[3] + f[4] - f[9] - f[10] - f[11] - f[12] - f[13];
    const R my = f[2] + f[6] + f[7] + f[8] + f[11] - f[0] - f[9] - f[15] - f[16] - f[17];
    const R mz = f[3] + f[5] + f[6] + f[12] + f[17] - f[1] - f[8] - f[10] - f[14] - f[15];
    den = r;
    if (div) {
        u = mx / r; w = my / r; v = mz / r;
    } else {
        const R ri = R(1) / r;
        u = mx * ri; w = my * ri; v = mz * ri;
    }
}

// prof_i / prof_j / prof_k (axis 0/1/2) at the two fixed coordinates c1, c2:
// out[4t + 0..3] = u, w (y), v (z), den of the t-th node, computed in R.
template <typename S, typename R>
__global__ void k_line(Lat<S, R> L, Geo g, int axis, int c1, int c2, double* out) {
    const int len = axis == 0 ? g.l : (axis == 1 ? g.m : g.n);
    const int t = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (t > len) return;
    const int i = axis == 0 ? t : c1, j = axis == 1 ? t : (axis == 0 ? c1 : c2), k = axis == 2 ? t : c2;
    R den, u, w, v;
    ref_macro(L, g.lin(i, j, k), true, den, u, w, v);
    out[4 * (t - 1) + 0] = (double)u;
    out[4 * (t - 1) + 1] = (double)w;
    out[4 * (t - 1) + 2] = (double)v;
    out[4 * (t - 1) + 3] = (double)den;
}

// One block per plane normal to `axis` (CODE/SRC/varm.F90:42-98 for axis z):
// FP64 sums of u, w, v (momentum times 1/den in R) and den over the plane's
// nodes, a fixed thread assignment and tree, then divided by the node count.
template <typename S, typename R>
__global__ void k_plane_means(Lat<S, R> L, Geo g, int axis, double* out) {
    const int pl = blockIdx.x;  // 0-based plane
    const int64_t cnt = axis == 0 ? (int64_t)g.m * g.n : (axis == 1 ? (int64_t)g.l * g.n : g.lm);
    double s[4] = {0, 0, 0, 0};
    for (int64_t t = threadIdx.x; t < cnt; t += blockDim.x) {
        int64_t lin;
        if (axis == 2) lin = (int64_t)pl * g.lm + t;
        else if (axis == 0) lin = pl + (int64_t)g.l * t;                             // t = (j-1) + m (k-1)
        else lin = (t % g.l) + (int64_t)g.l * (pl + (int64_t)g.m * (t / g.l));       // t = (i-1) + l (k-1)
        R den, u, w, v;
        ref_macro(L, lin, false, den, u, w, v);
        s[0] += (double)u; s[1] += (double)w; s[2] += (double)v; s[3] += (double)den;
    }
    __shared__ double sh[32][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 4; ++c)
        for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_down_sync(0xffffffffu, s[c], o);
    if (lane == 0)
        for (int c = 0; c < 4; ++c) sh[warp][c] = s[c];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int c = 0; c < 4; ++c) {
            double a = 0.0;
            for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) a += sh[wv][c];
            out[4 * pl + c] = a / (double)cnt;
        }
}

// Non-equilibrium stresses xx and xy of one node, CODE/SRC/flux_X.F90:162-240
// and CODE/SRC/flux_Y.F90, in R and the reference's expression order.
template <typename S, typename R>
__device__ __forceinline__ void ref_stress(const Lat<S, R>& L, int64_t lin, R omega, R& sxx, R& sxy) {
    R f[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = Store<S, R>::load(L.pop[q][lin], q, L.inv_scale);
    const R one = R(1), rf = R(3), qf = R(1.5), tre = R(3);
    const R p1 = Const<R>::p1(), p2 = Const<R>::p2();
    const R rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] +
                  f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    const R rhoinv = one / rho;
    const R xj = (f[0] + f[1] + f[2] + f[3] + f[4] - f[9] - f[10] - f[11] - f[12] - f[13]) * rhoinv;
    const R yj = (f[2] + f[6] + f[7] + f[8] + f[11] - f[0] - f[9] - f[15] - f[16] - f[17]) * rhoinv;
    const R zj = (f[3] + f[5] + f[6] + f[12] + f[17] - f[1] - f[8] - f[10] - f[14] - f[15]) * rhoinv;
    const R cvsq = xj * xj + yj * yj + zj * zj;
    auto fe = [&](R w, R e, R sq) { return rho * w * (one + rf * e + qf * (tre * sq * sq - cvsq)); };
    const R e[18] = {fe(p2, xj - yj, xj - yj),  fe(p2, xj - zj, xj - zj),  fe(p2, xj + yj, xj + yj),
                     fe(p2, xj + zj, xj + zj),  fe(p1, xj, xj),            fe(p1, zj, zj),
                     fe(p2, yj + zj, yj + zj),  fe(p1, yj, yj),            fe(p2, yj - zj, yj - zj),
                     fe(p2, -xj - yj, xj + yj), fe(p2, -xj - zj, xj + zj), fe(p2, -xj + yj, xj - yj),
                     fe(p2, -xj + zj, xj - zj), fe(p1, -xj, xj),           fe(p1, -zj, zj),
                     fe(p2, -yj - zj, yj + zj), fe(p1, -yj, yj),           fe(p2, -yj + zj, yj - zj)};
    const R visc = one - R(0.5) * omega;
    R xx = -rho / rf, xy = R(0);
#pragma unroll
    for (int q = 0; q < 18; ++q) {
        const R fn = f[q] - e[q];
        xx = xx - visc * R(cx_of(q)) * R(cx_of(q)) * fn;
        xy = xy - visc * R(cx_of(q)) * R(cy_of(q)) * fn;
    }
    sxx = xx;
    sxy = xy;
}

// The four faces of a control volume, FP64 sums: face 0/1 x = i1/i2 (stress
// xx over j1..j2, k1..k2), face 2/3 y = j1/j2 (stress xy over i1..i2, k1..k2).
struct CvBox {
    int i1, i2, j1, j2, k1, k2;
};

template <typename S, typename R>
__global__ void k_cv_drag(Lat<S, R> L, Geo g, CvBox b, R omega, Reduce red, double* out) {
    const int64_t nx = (int64_t)(b.j2 - b.j1 + 1) * (b.k2 - b.k1 + 1);
    const int64_t ny = (int64_t)(b.i2 - b.i1 + 1) * (b.k2 - b.k1 + 1);
    const int64_t total = 2 * nx + 2 * ny;
    double s[4] = {0, 0, 0, 0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int face, i, j, k;
        if (t < 2 * nx) {
            face = (int)(t / nx);
            const int64_t r = t % nx;
            i = face ? b.i2 : b.i1;
            j = b.j1 + (int)(r % (b.j2 - b.j1 + 1));
            k = b.k1 + (int)(r / (b.j2 - b.j1 + 1));
        } else {
            const int64_t u = t - 2 * nx;
            face = 2 + (int)(u / ny);
            const int64_t r = u % ny;
            j = face == 3 ? b.j2 : b.j1;
            i = b.i1 + (int)(r % (b.i2 - b.i1 + 1));
            k = b.k1 + (int)(r / (b.i2 - b.i1 + 1));
        }
        R xx, xy;
        ref_stress(L, g.lin(i, j, k), omega, xx, xy);
        s[face] += face < 2 ? (double)xx : (double)xy;
    }
    block_reduce_store<4>(s, red, out);
}

// Population q of the seeded equilibrium state (init_eq.h) over the haloed
// node range, into a staging buffer laid out like one host array.
template <typename T>
__global__ void k_init_population(T* out, int q, int64_t total, double u_in, double amp, uint64_t seed) {
    for (int64_t L = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; L < total; L += (int64_t)gridDim.x * blockDim.x) {
        T f[19];
        init_node<T>(L, u_in, amp, seed, f);
        out[L] = f[q];
    }
}

template <typename S, typename R>
__global__ void k_probes(Lat<S, R> L, Geo g, int npts, const int32_t* ijk, double* out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    const int i = ijk[3 * p], j = ijk[3 * p + 1], k = ijk[3 * p + 2];
    double a[19];
    for (int q = 0; q < 19; ++q) a[q] = (double)lat_load(L, g, q, i, j, k);
    double rho = 0.0;
    for (int q = 0; q < 19; ++q) rho += a[q];
    out[4 * p] = rho;
    out[4 * p + 1] = (a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13]) / rho;
    out[4 * p + 2] = (a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17]) / rho;
    out[4 * p + 3] = (a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15]) / rho;
}

// ---- host layout <-> device layout ------------------------------------------------------
// Host values (T = float or double) into the lattice and the halo shell.  16-bit storage
// from double converts in double: f = w + D/scale is exact there, so a state downloaded as
// double and uploaded again keeps every bit of D (through float, deviations below 2^-6
// lose their low bits to the rounding of f).  A host value that is not finite sets bit q
// of *bad (the caller rejects the state).
template <typename S, typename R, typename T>
__global__ void k_scatter(Lat<S, R> L, Geo g, int q, const T* src, int64_t total, unsigned int* bad) {
    constexpr bool exact16 = DevStore<S>::value && sizeof(T) == 8;
    const int64_t L2 = g.l + 2, M2 = g.m + 2;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % L2), j = (int)((idx / L2) % M2), k = (int)(idx / (L2 * M2));
        if (!isfinite(src[idx])) atomicOr(bad, 1u << q);
        const R v = (R)src[idx];
        if (g.interior(i, j, k)) {
            if constexpr (exact16)
                L.pop[q][g.lin(i, j, k)] =
                    DevStore<S>::from_d(((double)src[idx] - (double)weight<float>(q)) * (double)L.scale);
            else
                L.pop[q][g.lin(i, j, k)] = Store<S, R>::store(v, q, L.scale);
        } else {
            L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)] = v;
        }
    }
}

// The lattice and halo shell as host values; 16-bit storage to double in double (exact).
template <typename S, typename R, typename T>
__global__ void k_gather(Lat<S, R> L, Geo g, int q, T* dst, int64_t total) {
    constexpr bool exact16 = DevStore<S>::value && sizeof(T) == 8;
    const int64_t L2 = g.l + 2, M2 = g.m + 2;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(idx % L2), j = (int)((idx / L2) % M2), k = (int)(idx / (L2 * M2));
        if constexpr (exact16) {
            if (g.interior(i, j, k)) {
                dst[idx] = (double)weight<float>(q) +
                           (double)DevStore<S>::to_f(L.pop[q][g.lin(i, j, k)]) * (double)L.inv_scale;
                continue;
            }
        }
        dst[idx] = (T)lat_load(L, g, q, i, j, k);
    }
}

// x-face copy of the current lattice (after an upload): one thread per (j,k).
template <typename S, typename R>
__global__ void k_fill_xface(Lat<S, R> L, Geo g) {
    // one thread per (side, q, j, k), j fastest: the stores are coalesced, and every load
    // (a column of the lattice, stride l) is in flight at once
    const int64_t mn = (int64_t)g.m * g.n;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 36 * mn) return;
    const int sq = (int)(t / mn);  // side * 18 + q
    const int64_t jk = t - sq * mn;
    const int side = sq / 18, q = sq - 18 * side;
    const int j = (int)(jk % g.m) + 1, k = (int)(jk / g.m) + 1;
    L.xface[xface_idx(g, side, q, j, k)] = lat_load(L, g, q, side ? g.l : 1, j, k);
}

unsigned grid_for(int64_t work, int tpb, unsigned cap = 148u * 16u) {
    int64_t b = (work + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

}  // namespace

// x-slab faces: pack the five populations leaving through column x = 1 (side 0,
// cx = -1: q 9..13) or x = l (side 1, cx = +1: q 0..4), halo rows j = 0, m+1
// and k = 0, n+1 included, as a later load returns them; unpack received
// planes into the x = 0 (side 0, q 0..4) or x = l+1 (side 1, q 9..13) halo.
template <typename S, typename R>
__global__ void k_pack_x(Lat<S, R> L, Geo g, int side, R* out) {
    const int64_t plane = (int64_t)(g.m + 2) * (g.n + 2);
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5 * plane) return;
    const int c = (int)(t / plane);
    const int64_t jk = t % plane;
    const int j = (int)(jk % (g.m + 2)), k = (int)(jk / (g.m + 2));
    const int q = side ? c : 9 + c;
    const int i = side ? g.l : 1;
    out[t] = bc_load(L, g, q, i, j, k);
}

// The rim of the x-face copy's plane messages: the five outgoing populations on the
// halo rows of each exchange face column (sides: bit 0 = x = 1, bit 1 = x = l), read
// after the halo kernels wrote them.
template <typename S, typename R>
__global__ void k_pack_x_rim(Lat<S, R> L, Geo g, int sides) {
    const int64_t per = g.xr / 5;  // halo-row nodes of one face plane
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * g.xr) return;
    const int side = (int)(t / g.xr);
    if (!((sides >> side) & 1)) return;
    const int64_t r = t - side * g.xr;
    const int c = (int)(r / per);
    int j, k;
    xface_rim_node(g, r - c * per, &j, &k);
    const int q = side ? c : 9 + c;
    L.xface[xface_rim_offset(g, side) + r] = lat_load(L, g, q, side ? g.l : 1, j, k);
}

// A received plane message into the x = 0 (side 0, q 0..4) or x = l+1 (side 1,
// q 9..13) halo plane.  It left the neighbour's opposite side: into side 0 come
// the five m*n blocks then the rim, into side 1 the rim then the blocks.
template <typename S, typename R>
__global__ void k_unpack_x_view(Lat<S, R> L, Geo g, int side, const R* in) {
    const int64_t mn = g.mn, per = g.xr / 5;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5 * mn + g.xr) return;
    const int64_t b = side ? t - g.xr : t;  // position among the blocks (< 0: on the rim)
    int c, j, k;
    if (b >= 0 && b < 5 * mn) {
        c = (int)(b / mn);
        const int64_t jk = b - c * mn;
        j = (int)(jk % g.m) + 1;
        k = (int)(jk / g.m) + 1;
    } else {
        const int64_t r = side ? t : t - 5 * mn;
        c = (int)(r / per);
        xface_rim_node(g, r - c * per, &j, &k);
    }
    const int q = side ? 9 + c : c;
    const int i = side ? g.l + 1 : 0;
    L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)] = in[t];
}

template <typename S, typename R>
__global__ void k_unpack_x(Lat<S, R> L, Geo g, int side, const R* in) {
    const int64_t plane = (int64_t)(g.m + 2) * (g.n + 2);
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 5 * plane) return;
    const int c = (int)(t / plane);
    const int64_t jk = t % plane;
    const int j = (int)(jk % (g.m + 2)), k = (int)(jk / (g.m + 2));
    const int q = side ? 9 + c : c;
    const int i = side ? g.l + 1 : 0;
    L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)] = in[t];
}

template <typename S, typename R>
void launch_pack_x(const Lat<S, R>& L, const Geo& g, int side, R* out, cudaStream_t st) {
    const int64_t work = 5 * (int64_t)(g.m + 2) * (g.n + 2);
    k_pack_x<S, R><<<(unsigned)((work + kTpb - 1) / kTpb), kTpb, 0, st>>>(L, g, side, out);
}

template <typename S, typename R>
void launch_pack_x_rim(const Lat<S, R>& L, const Geo& g, int sides, cudaStream_t st) {
    const int64_t work = 2 * g.xr;
    k_pack_x_rim<S, R><<<(unsigned)((work + kTpb - 1) / kTpb), kTpb, 0, st>>>(L, g, sides);
}

template <typename S, typename R>
void launch_unpack_x_view(const Lat<S, R>& L, const Geo& g, int side, const R* in, cudaStream_t st) {
    const int64_t work = 5 * (int64_t)(g.m + 2) * (g.n + 2);
    k_unpack_x_view<S, R><<<(unsigned)((work + kTpb - 1) / kTpb), kTpb, 0, st>>>(L, g, side, in);
}

template <typename S, typename R>
void launch_unpack_x(const Lat<S, R>& L, const Geo& g, int side, const R* in, cudaStream_t st) {
    const int64_t work = 5 * (int64_t)(g.m + 2) * (g.n + 2);
    k_unpack_x<S, R><<<(unsigned)((work + kTpb - 1) / kTpb), kTpb, 0, st>>>(L, g, side, in);
}

template <typename S, typename R>
int launch_bc_fused(const Lat<S, R>& L, const Geo& g, const int bc[6], const Phys<R>& ph, unsigned int* bar,
                    cudaStream_t st) {
    const int l = g.l, m = g.m, n = g.n;
    BcPlan<R> plan;
    plan.n = 0;
    plan.u_inflow = ph.u_inflow;
    plan.force = ph.force;
    auto add = [&](int kind, int flag, Range2 r) { plan.ph[plan.n++] = BcPhase{kind, flag, r}; };
    if (bc[0] != 6) {
        const int f = bc[0];
        add(kBcFront, f, (f == 0) ? Range2{0, m + 1, 1, n} : Range2{1, m, 1, n});
        if (f == 5) add(kBcFrontFix, 0, Range2{0, (m > n ? m : n) + 1, 0, 2});
    }
    if (bc[1] != 6) {
        const int f = bc[1];
        add(kBcRear, f, (f == 0) ? Range2{0, m + 1, 1, n} : (f == 1) ? Range2{1, m, 1, n} : Range2{0, m + 2, 0, n + 2});
    }
    add(kBcUp, bc[4], (bc[4] == 3) ? Range2{0, l + 2, 0, m + 2} : Range2{1, l, 1, m});
    add(kBcDown, bc[5], Range2{1, l, 1, m});
    add(kBcLeft, bc[3], (bc[3] == 0) ? Range2{0, l + 1, 1, n} : Range2{1, l, 1, n});
    add(kBcRight, bc[2], (bc[2] == 0) ? Range2{0, l + 1, 1, n} : Range2{1, l, 1, n});
    const int fixes = ((bc[3] == 3 && bc[4] == 3) ? 1 : 0) | ((bc[2] == 3 && bc[4] == 3) ? 2 : 0) |
                      ((bc[2] == 3 && bc[5] == 3) ? 4 : 0) | ((bc[3] == 3 && bc[5] == 3) ? 8 : 0);
    if (fixes) add(kBcEdgeFix, fixes, Range2{1, l, 0, 1});
    int64_t need = 1;
    for (int p = 0; p < plan.n; ++p) need = std::max<int64_t>(need, (plan.ph[p].r.size() + kTpb - 1) / kTpb);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kBcMaxDevices) return -1;
    const int cap = g_bc_fused_blocks[dev][bc_type_index<S>()];
    if (!g_bc_fused_ok[dev] || cap <= 0) return -1;
    unsigned grid = (unsigned)std::min<int64_t>(need, cap);
    Lat<S, R> Lc = L;
    Geo gc = g;
    void* args[] = {&Lc, &gc, &plan, &bar};
    if (cudaLaunchCooperativeKernel((const void*)k_bc_all<S, R>, dim3(grid), dim3(kTpb), args, 0, st) != cudaSuccess)
        return -1;
    return 1;
}

template <typename S, typename R>
int launch_bc(const Lat<S, R>& L, const Geo& g, const int bc[6], const Phys<R>& ph, cudaStream_t st,
              unsigned int* bar) {
    if (bar) {  // one cooperative launch for all blocks when the device allows it
        const int n = launch_bc_fused<S, R>(L, g, bc, ph, bar, st);
        if (n > 0) return n;
        cudaGetLastError();  // a refused cooperative launch leaves nothing behind: use one launch per block
    }
    const int l = g.l, m = g.m, n = g.n;
    int launches = 4;
    // front (an x-slab exchange face gets its plane from the neighbour instead)
    if (bc[0] != 6) {
        ++launches;
        const int f = bc[0];
        Range2 r = (f == 0) ? Range2{0, m + 1, 1, n} : Range2{1, m, 1, n};
        k_front<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, f);
        if (f == 5) {
            Range2 rf{0, (m > n ? m : n) + 1, 0, 2};
            k_front_fix<S, R><<<rf.blocks(kTpb), kTpb, 0, st>>>(L, g, rf);
            ++launches;
        }
    }
    // rear
    if (bc[1] != 6) {
        ++launches;
        const int f = bc[1];
        Range2 r = (f == 0) ? Range2{0, m + 1, 1, n} : (f == 1) ? Range2{1, m, 1, n} : Range2{0, m + 2, 0, n + 2};
        k_rear<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, f, ph.u_inflow);
    }
    // up
    {
        const int f = bc[4];
        Range2 r = (f == 3) ? Range2{0, l + 2, 0, m + 2} : Range2{1, l, 1, m};
        k_up<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, f, ph.force);
    }
    // down
    {
        Range2 r{1, l, 1, m};
        k_down<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, bc[5]);
    }
    // left
    {
        const int f = bc[3];
        Range2 r = (f == 0) ? Range2{0, l + 1, 1, n} : Range2{1, l, 1, n};
        k_left<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, f);
    }
    // right
    {
        const int f = bc[2];
        Range2 r = (f == 0) ? Range2{0, l + 1, 1, n} : Range2{1, l, 1, n};
        k_right<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, f);
    }
    const int fixes = ((bc[3] == 3 && bc[4] == 3) ? 1 : 0) | ((bc[2] == 3 && bc[4] == 3) ? 2 : 0) |
                      ((bc[2] == 3 && bc[5] == 3) ? 4 : 0) | ((bc[3] == 3 && bc[5] == 3) ? 8 : 0);
    if (fixes) {
        Range2 r{1, l, 0, 1};
        k_edge_fix<S, R><<<r.blocks(kTpb), kTpb, 0, st>>>(L, g, r, fixes);
        ++launches;
    }
    return launches;
}

template <typename S, typename R>
void launch_bounce_drag(const Lat<S, R>& L, const Geo& g, const int bc[6], const int32_t* list,
                        const uint64_t* links, int64_t nlist, bool do_bounce, const Reduce& red, double* series,
                        int64_t cap, int64_t* d_itime, bool advance, cudaStream_t st) {
    const int per_x = (bc[0] == 0 && bc[1] == 0), per_y = (bc[2] == 0 && bc[3] == 0);
    const int per_z = (bc[4] == 0 && bc[5] == 0);
    const unsigned blocks = grid_for(nlist, kTpb, (unsigned)red.max_blocks);
    k_bounce_drag<S, R><<<blocks, kTpb, 0, st>>>(L, g, per_x, per_y, per_z, list, links, nlist, do_bounce ? 1 : 0,
                                                 red, series, cap, d_itime, advance ? 1 : 0);
}

template <typename S, typename R>
void launch_fill_xface(const Lat<S, R>& L, const Geo& g, cudaStream_t st) {
    const int64_t work = 36 * (int64_t)g.m * g.n;
    k_fill_xface<S, R><<<(unsigned)((work + kTpb - 1) / kTpb), kTpb, 0, st>>>(L, g);
}

template <typename S, typename R>
void launch_monitor(const Lat<S, R>& L, const Geo& g, const Mask& mk, const Reduce& red, double* out,
                    cudaStream_t st) {
    const unsigned blocks = grid_for(g.N, kTpb, (unsigned)red.max_blocks);
    k_monitor<S, R><<<blocks, kTpb, 0, st>>>(L, g, mk, red, out);
}

template <typename S, typename R>
void launch_region_sums(const Lat<S, R>& L, const Geo& g, const Mask& mk, const uint8_t* region, const Reduce& red,
                        double* out, cudaStream_t st) {
    const unsigned blocks = grid_for(g.N, kTpb, (unsigned)red.max_blocks);
    k_region_sums<S, R><<<blocks, kTpb, 0, st>>>(L, g, mk, region, red, out);
}

template <typename S, typename R>
void launch_line(const Lat<S, R>& L, const Geo& g, int axis, int c1, int c2, double* out, cudaStream_t st) {
    const int len = axis == 0 ? g.l : (axis == 1 ? g.m : g.n);
    k_line<S, R><<<(len + 127) / 128, 128, 0, st>>>(L, g, axis, c1, c2, out);
}

template <typename S, typename R>
void launch_plane_means(const Lat<S, R>& L, const Geo& g, int axis, double* out, cudaStream_t st) {
    const int len = axis == 0 ? g.l : (axis == 1 ? g.m : g.n);
    k_plane_means<S, R><<<len, 256, 0, st>>>(L, g, axis, out);
}

template <typename S, typename R>
void launch_cv_drag(const Lat<S, R>& L, const Geo& g, const int box[6], R omega, const Reduce& red, double* out,
                    cudaStream_t st) {
    const CvBox b{box[0], box[1], box[2], box[3], box[4], box[5]};
    const int64_t total = 2 * (int64_t)(b.j2 - b.j1 + 1) * (b.k2 - b.k1 + 1) +
                          2 * (int64_t)(b.i2 - b.i1 + 1) * (b.k2 - b.k1 + 1);
    k_cv_drag<S, R><<<grid_for(total, kTpb, (unsigned)red.max_blocks), kTpb, 0, st>>>(L, g, b, omega, red, out);
}

template <typename T>
void launch_init_population(T* staging, const Geo& g, int q, double u_in, double amp, uint64_t seed, cudaStream_t st) {
    const int64_t total = (int64_t)(g.l + 2) * (g.m + 2) * (g.n + 2);
    k_init_population<T><<<grid_for(total, kTpb), kTpb, 0, st>>>(staging, q, total, u_in, amp, seed);
}
template void launch_init_population<float>(float*, const Geo&, int, double, double, uint64_t, cudaStream_t);
template void launch_init_population<double>(double*, const Geo&, int, double, double, uint64_t, cudaStream_t);

template <typename S, typename R>
void launch_probes(const Lat<S, R>& L, const Geo& g, int npts, const int32_t* ijk, double* out,
                   cudaStream_t st) {
    k_probes<S, R><<<(npts + 127) / 128, 128, 0, st>>>(L, g, npts, ijk, out);
}

template <typename S, typename R, typename T>
void launch_scatter(const Lat<S, R>& L, const Geo& g, int q, const T* staging, unsigned int* bad, cudaStream_t st) {
    const int64_t total = (int64_t)(g.l + 2) * (g.m + 2) * (g.n + 2);
    k_scatter<S, R, T><<<grid_for(total, kTpb), kTpb, 0, st>>>(L, g, q, staging, total, bad);
}

template <typename S, typename R, typename T>
void launch_gather(const Lat<S, R>& L, const Geo& g, int q, T* staging, cudaStream_t st) {
    const int64_t total = (int64_t)(g.l + 2) * (g.m + 2) * (g.n + 2);
    k_gather<S, R, T><<<grid_for(total, kTpb), kTpb, 0, st>>>(L, g, q, staging, total);
}

#define EUP_INST(S, R)                                                                                 \
    template int launch_bc<S, R>(const Lat<S, R>&, const Geo&, const int*, const Phys<R>&, cudaStream_t,   \
                                 unsigned int*);                                                          \
    template void launch_bounce_drag<S, R>(const Lat<S, R>&, const Geo&, const int*, const int32_t*,   \
                                           const uint64_t*, int64_t, bool, const Reduce&, double*,     \
                                           int64_t, int64_t*, bool, cudaStream_t);                     \
    template void launch_fill_xface<S, R>(const Lat<S, R>&, const Geo&, cudaStream_t);                 \
    template void launch_pack_x<S, R>(const Lat<S, R>&, const Geo&, int, R*, cudaStream_t);              \
    template void launch_unpack_x<S, R>(const Lat<S, R>&, const Geo&, int, const R*, cudaStream_t);      \
    template void launch_pack_x_rim<S, R>(const Lat<S, R>&, const Geo&, int, cudaStream_t);              \
    template void launch_unpack_x_view<S, R>(const Lat<S, R>&, const Geo&, int, const R*, cudaStream_t); \
    template void launch_line<S, R>(const Lat<S, R>&, const Geo&, int, int, int, double*, cudaStream_t);   \
    template void launch_plane_means<S, R>(const Lat<S, R>&, const Geo&, int, double*, cudaStream_t);     \
    template void launch_cv_drag<S, R>(const Lat<S, R>&, const Geo&, const int*, R, const Reduce&, double*, \
                                       cudaStream_t);                                                     \
    template void launch_region_sums<S, R>(const Lat<S, R>&, const Geo&, const Mask&, const uint8_t*,   \
                                           const Reduce&, double*, cudaStream_t);                         \
    template void launch_monitor<S, R>(const Lat<S, R>&, const Geo&, const Mask&, const Reduce&,       \
                                       double*, cudaStream_t);                                         \
    template void launch_probes<S, R>(const Lat<S, R>&, const Geo&, int, const int32_t*, double*,      \
                                      cudaStream_t);                                                   \
    template void launch_scatter<S, R, float>(const Lat<S, R>&, const Geo&, int, const float*,         \
                                              unsigned int*, cudaStream_t);                            \
    template void launch_scatter<S, R, double>(const Lat<S, R>&, const Geo&, int, const double*,       \
                                               unsigned int*, cudaStream_t);                           \
    template void launch_gather<S, R, float>(const Lat<S, R>&, const Geo&, int, float*, cudaStream_t); \
    template void launch_gather<S, R, double>(const Lat<S, R>&, const Geo&, int, double*, cudaStream_t);

EUP_INST(float, float)
EUP_INST(double, double)
EUP_INST(__half, float)
EUP_INST(__nv_bfloat16, float)

cudaError_t prepare_bc_fused(unsigned int* bar) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kBcMaxDevices) return cudaSuccess;  // separate launches there
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    int coop = 0;
    if ((e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev)) != cudaSuccess) return e;
    const void* ks[4] = {(const void*)k_bc_all<float, float>, (const void*)k_bc_all<double, double>,
                         (const void*)k_bc_all<__half, float>, (const void*)k_bc_all<__nv_bfloat16, float>};
    for (int t = 0; t < 4; ++t) {
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ks[t], kTpb, 0)) != cudaSuccess) return e;
        g_bc_fused_blocks[dev][t] = per_sm * sms;
    }
    if (!coop) return cudaSuccess;
    // a cooperative launch must survive stream capture (every step runs as a CUDA graph):
    // capture one on a private stream, instantiate and run the graph once
    cudaStream_t s = nullptr;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return e;
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    void* args[] = {&bar};
    const bool launched =
        ok && cudaLaunchCooperativeKernel((const void*)k_coop_probe, dim3(2), dim3(32), args, 0, s) == cudaSuccess;
    cudaGraph_t graph = nullptr;
    ok = (cudaStreamEndCapture(s, &graph) == cudaSuccess) && launched && graph;
    cudaGraphExec_t exec = nullptr;
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (ok) ok = cudaGraphLaunch(exec, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
    unsigned int word[3] = {1, 0, 1};
    if (ok) ok = cudaMemcpy(word, bar, sizeof(word), cudaMemcpyDeviceToHost) == cudaSuccess;
    // the probe's two CTAs met at the barrier: no timeout, arrivals back to zero, one generation
    ok = ok && word[0] == 0 && word[1] == 1 && word[2] == 0;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamDestroy(s);
    cudaGetLastError();
    g_bc_fused_ok[dev] = ok;
    return cudaMemset(bar, 0, 3 * sizeof(unsigned int));
}

}  // namespace eup

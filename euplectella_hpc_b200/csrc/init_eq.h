// Seeded equilibrium initial state, shared by the host initialiser and the
// device one so that both produce the same bits: node L of the haloed arrays
// (i fastest, L = i + (l+2)(j + (m+2) k), 0-based) gets the equilibrium of
// CODE/SRC/init.F90:194-232 at rho = 1 and u = (u_in + amp xi_0, amp xi_1,
// amp xi_2), xi_c uniform in [-1, 1) from splitmix64(seed + 3L + c).
// Neither side contracts a multiply and an add (the device code is compiled
// with --fmad=false, the host code for a target without fused multiply-add).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define EUP_HD __host__ __device__
#else
#define EUP_HD
#endif

namespace eup {

EUP_HD inline uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Equilibrium of CODE/SRC/init.F90:194-232 for one node, in type T.
template <typename T>
EUP_HD inline void equilibrium(T xj, T yj, T zj, T out[19]) {
    const T rf = T(3), qf = T(1.5), t3 = T(3), one = T(1), crho = T(1);
    const T p0 = (T)(1.0 / 3.0), p1 = (T)(1.0 / 18.0), p2 = (T)(1.0 / 36.0);
    const T cvsq = xj * xj + yj * yj + zj * zj;
    const T c[19] = {
        rf * (xj - yj) + qf * (t3 * (xj - yj) * (xj - yj) - cvsq),
        rf * (xj - zj) + qf * (t3 * (xj - zj) * (xj - zj) - cvsq),
        rf * (xj + yj) + qf * (t3 * (xj + yj) * (xj + yj) - cvsq),
        rf * (xj + zj) + qf * (t3 * (xj + zj) * (xj + zj) - cvsq),
        rf * (xj) + qf * (t3 * (xj) * (xj) - cvsq),
        rf * (zj) + qf * (t3 * (zj) * (zj) - cvsq),
        rf * (yj + zj) + qf * (t3 * (yj + zj) * (yj + zj) - cvsq),
        rf * (yj) + qf * (t3 * (yj) * (yj) - cvsq),
        rf * (yj - zj) + qf * (t3 * (yj - zj) * (yj - zj) - cvsq),
        rf * (-xj - yj) + qf * (t3 * (xj + yj) * (xj + yj) - cvsq),
        rf * (-xj - zj) + qf * (t3 * (xj + zj) * (xj + zj) - cvsq),
        rf * (-xj + yj) + qf * (t3 * (xj - yj) * (xj - yj) - cvsq),
        rf * (-xj + zj) + qf * (t3 * (xj - zj) * (xj - zj) - cvsq),
        rf * (-xj) + qf * (t3 * (xj) * (xj) - cvsq),
        rf * (-zj) + qf * (t3 * (zj) * (zj) - cvsq),
        rf * (-yj - zj) + qf * (t3 * (yj + zj) * (yj + zj) - cvsq),
        rf * (-yj) + qf * (t3 * (yj) * (yj) - cvsq),
        rf * (-yj + zj) + qf * (t3 * (yj - zj) * (yj - zj) - cvsq),
        rf * (T(0)) + qf * (t3 * (T(0)) * (T(0)) - cvsq),
    };
    for (int q = 0; q < 19; ++q) {
        const int wc = (q == 18) ? 0 : (q == 4 || q == 5 || q == 7 || q == 13 || q == 14 || q == 16) ? 1 : 2;
        const T w = wc == 0 ? p0 : (wc == 1 ? p1 : p2);
        out[q] = crho * w * (one + c[q]);
    }
}

// The 19 initial populations of haloed node L.
template <typename T>
EUP_HD inline void init_node(int64_t L, double u_in, double amp, uint64_t seed, T f[19]) {
    double xi[3];
    for (int c = 0; c < 3; ++c) {
        const uint64_t h = splitmix64(seed + 3u * (uint64_t)L + (uint64_t)c);
        xi[c] = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
    equilibrium<T>((T)(u_in + amp * xi[0]), (T)(amp * xi[1]), (T)(amp * xi[2]), f);
}

}  // namespace eup

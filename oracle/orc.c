/*
 * oracle/orc.c -- CPU ORACLE (test infrastructure only; see orc.h).
 * Instantiates the restatement in orc_impl.h for float (the reference's
 * default mykind = sp, CODE/SRC/precision.F90:26) and double (-DDOUBLE_P).
 */
#include "orc.h"

#include <math.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* splitmix64 output for state x (Steele, Lea, Flood 2014). */
uint64_t orc_splitmix64(uint64_t x)
{
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int32_t orc_nthreads(void)
{
#ifdef _OPENMP
    return (int32_t)omp_get_max_threads();
#else
    return 1;
#endif
}

#define REAL float
#define P f
#define RSIN sinf
#define RCOS cosf
#include "orc_impl.h"
#undef REAL
#undef P
#undef RSIN
#undef RCOS

#define REAL double
#define P d
#define RSIN sin
#define RCOS cos
#include "orc_impl.h"
#undef REAL
#undef P
#undef RSIN
#undef RCOS

/* D3Q19 velocities in the reference's order a01..a18 (CODE/SRC/bgk3d.F90:30-49). */
static const int CX[18] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0};
static const int CY[18] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1};
static const int CZ[18] = {0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1};

static int solid_at(const orc_params* p, const int32_t* obs, int i, int j, int k)
{
    const int l = p->l, m = p->m, n = p->n;
    if (i < 1 || i > l || j < 1 || j > m || k < 1 || k > n) return 0;
    return OBS(i, j, k) == 1;
}

/*
 * Link classification per interior node (interior order, i fastest):
 * bit q-1 (q = 1..18) is set when the node is fluid and its upstream
 * neighbour x - c_q is an interior solid voxel, i.e. the population the pull
 * of CODE/SRC/movef.F90:48-65 brings in was written by the bounce-back of
 * CODE/SRC/bcond.obs.F90:56-73.  Bit 31 marks a solid node.
 */
void orc_links(const orc_params* p, const int32_t* obs, uint32_t* links)
{
    const int l = p->l, m = p->m, n = p->n;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const int64_t o = (int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1));
                uint32_t w = 0;
                if (OBS(i, j, k) == 1) {
                    w = 0x80000000u;
                } else {
                    for (int q = 0; q < 18; ++q)
                        if (solid_at(p, obs, i - CX[q], j - CY[q], k - CZ[q])) w |= 1u << q;
                }
                links[o] = w;
            }
}

/*
 * Solid voxels that can hand a value to the fluid: solid with at least one of
 * the 18 neighbours not an interior solid voxel (fluid or halo).  Only these
 * values of CODE/SRC/bcond.obs.F90 are ever read by a fluid node or a halo
 * plane.  Returns the count; list (may be NULL) gets interior linear indices
 * in ascending order.
 */
int64_t orc_boundary_solid(const orc_params* p, const int32_t* obs, int64_t* list)
{
    const int l = p->l, m = p->m, n = p->n;
    int64_t cnt = 0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                if (OBS(i, j, k) != 1) continue;
                int open = 0;
                for (int q = 0; q < 18 && !open; ++q)
                    if (!solid_at(p, obs, i + CX[q], j + CY[q], k + CZ[q])) open = 1;
                if (!open) continue;
                if (list) list[cnt] = (int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1));
                ++cnt;
            }
    return cnt;
}

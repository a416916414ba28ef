/*
 * oracle/orc.h -- CPU ORACLE for the D3Q19 BGK time step (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of giacomofalcucci/Euplectella_HPC's serial
 * build (`-DSERIAL -DORIGINAL -DOBSTACLES`), written from the reference's
 * Fortran sources.  It is the checker for the CUDA path and the timed CPU
 * baseline; it is never linked into, or called by, the product library.
 *
 * PARITY STATUS: parity unpinned.  The reference ships no tests, golden
 * vectors or fixtures, and it cannot be built here (no Fortran compiler), so
 * this restatement is pinned only by analytic known-answer tests (rest state,
 * uniform periodic flow, mass conservation, hand-evaluated equilibria,
 * bounce-back symmetry) and by fixtures it generated itself.
 *
 * Layout: exactly the reference's.  Each population is one haloed 3-D array
 * a_q(0:l+1, 0:m+1, 0:n+1), Fortran order (i fastest), as allocated in
 * CODE/SRC/alloca.F90:94-132.  Population order q = 1..19 follows the
 * reference's a01..a19 (velocity table CODE/SRC/bgk3d.F90:30-49); in C the
 * index is q-1.  `obs` is obs(1:l,1:m,1:n), 1 = solid (CODE/SRC/alloca.F90:91).
 *
 * Boundary flag codes per face are the reference's (CODE/SRC/build.bcond.F90:11-17):
 *   0 periodic, 1 no-slip, 2 lid (up only), 3 free-slip, 4 inflow (rear only),
 *   5 outflow (front only).
 * Face order in bc[6]: front (x=l+1), rear (x=0), right (y=m+1), left (y=0),
 * up (z=n+1), down (z=0).
 */
#ifndef EUP_ORACLE_H
#define EUP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FRONT = 0, ORC_REAR = 1, ORC_RIGHT = 2, ORC_LEFT = 3, ORC_UP = 4, ORC_DOWN = 5 };

typedef struct orc_params {
    int32_t l, m, n;      /* interior sizes (serial: l=lx, m=ly, n=lz) */
    int32_t bc[6];        /* reference flag per face, order above */
    double svisc;         /* kinematic viscosity, rounded to REAL first (namelist read) */
    double u0;            /* body-force velocity scale (0 when there is an inlet) */
    double u_inflow;      /* inlet velocity (CODE/SRC/build.bcond.F90:321) */
    double u00;           /* lid velocity scale, force = u00/6 (CODE/SRC/bcond.bc.F90:50-56) */
} orc_params;

/* Per-precision entry points: orc_f_* (REAL=float), orc_d_* (REAL=double). */
#define ORC_DECLARE(P, REAL)                                                              \
    void orc_##P##_constants(const orc_params* p, REAL* omega, REAL* fgrad);              \
    void orc_##P##_bcond_obs(const orc_params* p, REAL* const a[19], const int32_t* obs); \
    void orc_##P##_bcond_bc(const orc_params* p, REAL* const a[19]);                      \
    void orc_##P##_movef(const orc_params* p, REAL* const a[19], REAL* const b[19]);      \
    void orc_##P##_col(const orc_params* p, REAL* const a[19], REAL* const b[19]);        \
    int orc_##P##_run(const orc_params* p, REAL* const a[19], REAL* const b[19],          \
                      const int32_t* obs, int32_t nsteps);                                \
    void orc_##P##_init_perturbed(int32_t l, int32_t m, int32_t n, double u_in,           \
                                  double amp, uint64_t seed, REAL* const a[19]);          \
    int orc_##P##_init_reference(int32_t opt, int32_t l, int32_t m, int32_t n,            \
                                 const int32_t glob[3], const int32_t start[3],           \
                                 int32_t periodic, double u0, REAL* const a[19]);         \
    void orc_##P##_mem_force(const orc_params* p, REAL* const a[19], const int32_t* obs,  \
                             double out[3]);                                              \
    void orc_##P##_monitor(const orc_params* p, REAL* const a[19], const int32_t* obs,    \
                           double out[5]);                                                \
    void orc_##P##_macro(const orc_params* p, REAL* const a[19], double* rho,             \
                         double* ux, double* uy, double* uz);                             \
    void orc_##P##_line(const orc_params* p, REAL* const a[19], int32_t axis, int32_t c1, \
                        int32_t c2, double* out);                                         \
    void orc_##P##_plane_means(const orc_params* p, REAL* const a[19], int32_t axis,      \
                               double* out);                                              \
    void orc_##P##_cv_drag(const orc_params* p, REAL* const a[19], const int32_t box[6],  \
                           double out[2]);

ORC_DECLARE(f, float)
ORC_DECLARE(d, double)

/* The synthetic bodies of the benchmark workloads (orc_geom.c): obs (n, m, l),
 * 1 = solid, bit-identical to the product's voxelisers; return the solid count. */
int64_t orc_voxelise_shell(int32_t l, int32_t m, int32_t n, double x0, double length, double yc, double zc,
                           double outer_d, double strut_d, double pitch, uint64_t seed, int32_t* obs);
int64_t orc_voxelise_cylinder_z(int32_t l, int32_t m, int32_t n, double xc, double yc, double r, int32_t* obs);

/* Precision-independent helpers. */
void orc_links(const orc_params* p, const int32_t* obs, uint32_t* links);
int64_t orc_boundary_solid(const orc_params* p, const int32_t* obs, int64_t* list);
uint64_t orc_splitmix64(uint64_t x);
int32_t orc_nthreads(void);

#ifdef __cplusplus
}
#endif
#endif

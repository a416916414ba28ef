/*
 * oracle/orc_impl.h -- body of the CPU ORACLE (test infrastructure), included
 * once per precision by oracle/orc.c with REAL and P defined.  Every routine
 * cites the reference routine (path within giacomofalcucci/Euplectella_HPC) it
 * restates.  Arithmetic keeps the reference's expression grouping and
 * left-to-right evaluation so that an IEEE implementation without contraction
 * reproduces it bit for bit (the file is compiled with -ffp-contract=off).
 */
#define CAT_(a, b, c) a##b##c
#define CAT(a, b, c) CAT_(a, b, c)
#define FN(name) CAT(orc_, P, _##name)

/* Haloed index: a_q(i,j,k) with i in 0..l+1 (CODE/SRC/alloca.F90:94-132). */
#define IDX(i, j, k) ((int64_t)(i) + L2 * ((int64_t)(j) + M2 * (int64_t)(k)))
#define A(q, i, j, k) a[(q) - 1][IDX(i, j, k)]
#define B(q, i, j, k) b[(q) - 1][IDX(i, j, k)]
/* obs(1:l,1:m,1:n) */
#define OBS(i, j, k) obs[((int64_t)(i) - 1) + (int64_t)l * (((int64_t)(j) - 1) + (int64_t)m * ((int64_t)(k) - 1))]

#define DECL_SIZES(p)                          \
    const int l = (p)->l, m = (p)->m, n = (p)->n; \
    const int l1 = l + 1, m1 = m + 1, n1 = n + 1; \
    const int64_t L2 = l + 2, M2 = m + 2;         \
    (void)l1; (void)m1; (void)n1; (void)L2; (void)M2

/* Lattice constants, CODE/SRC/storage.F90:54-81,194-205: computed in a wider
 * kind and rounded to mykind. */
#define RF ((REAL)3.0)
#define QF ((REAL)1.5)
#define UNO ((REAL)1.0)
#define TRE ((REAL)3.0)
#define ZERO ((REAL)0.0)
#define P0 ((REAL)(1.0 / 3.0))
#define P1 ((REAL)(1.0 / 18.0))
#define P2 ((REAL)(1.0 / 36.0))

/* omega and the body force, CODE/SRC/hencol.F90:30-39 (SERIAL branch). */
void FN(constants)(const orc_params* p, REAL* omega, REAL* fgrad)
{
    const REAL svisc = (REAL)p->svisc; /* namelist value held as real(mykind) */
    const REAL u0 = (REAL)p->u0;
    *omega = (REAL)(2.0 / (6.0 * (double)svisc + 1.0));
    /* fgrad = 4.0*u0*svisc/(5.0*real(n)*real(n)), all operands real(mykind) */
    *fgrad = (REAL)4.0 * u0 * svisc / ((REAL)5.0 * (REAL)p->n * (REAL)p->n);
}

/*
 * Halfway bounce-back on solid voxels, CODE/SRC/bcond.obs.F90:47-77:
 * a_q(x) = a_opp(q)(x + c_q) for every solid x in the obstacle bounding box
 * (bbox from CODE/SRC/build.obs.F90:121-127), loops k, j, i ascending as in the
 * serial build.
 */
void FN(bcond_obs)(const orc_params* p, REAL* const a[19], const int32_t* obs)
{
    DECL_SIZES(p);
    int imin = l + 1, imax = 0, jmin = m + 1, jmax = 0, kmin = n + 1, kmax = 0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i)
                if (OBS(i, j, k) == 1) {
                    if (i < imin) imin = i;
                    if (i > imax) imax = i;
                    if (j < jmin) jmin = j;
                    if (j > jmax) jmax = j;
                    if (k < kmin) kmin = k;
                    if (k > kmax) kmax = k;
                }
    for (int k = kmin; k <= kmax; ++k)
        for (int j = jmin; j <= jmax; ++j)
            for (int i = imin; i <= imax; ++i) {
                if (OBS(i, j, k) != 1) continue;
                A(1, i, j, k) = A(12, i + 1, j - 1, k);
                A(2, i, j, k) = A(13, i + 1, j, k - 1);
                A(3, i, j, k) = A(10, i + 1, j + 1, k);
                A(4, i, j, k) = A(11, i + 1, j, k + 1);
                A(5, i, j, k) = A(14, i + 1, j, k);
                A(6, i, j, k) = A(15, i, j, k + 1);
                A(7, i, j, k) = A(16, i, j + 1, k + 1);
                A(8, i, j, k) = A(17, i, j + 1, k);
                A(9, i, j, k) = A(18, i, j + 1, k - 1);
                A(10, i, j, k) = A(3, i - 1, j - 1, k);
                A(11, i, j, k) = A(4, i - 1, j, k - 1);
                A(12, i, j, k) = A(1, i - 1, j + 1, k);
                A(13, i, j, k) = A(2, i - 1, j, k + 1);
                A(14, i, j, k) = A(5, i - 1, j, k);
                A(15, i, j, k) = A(6, i, j, k - 1);
                A(16, i, j, k) = A(7, i, j - 1, k - 1);
                A(17, i, j, k) = A(8, i, j - 1, k);
                A(18, i, j, k) = A(9, i, j - 1, k + 1);
            }
}

/*
 * Halo planes, CODE/SRC/bcond.bc.F90:22-1052 as compiled with -DSERIAL and
 * without the PERIODIC/CHANNEL/INLET/DUCT/CHECK2D/MIXING/FREESLIP/SPONGES
 * presets (flags set directly).  Blocks run in the reference's order: front,
 * rear, up, down, left, right, then the free-slip edge fixes.  Under SERIAL
 * every periodic face satisfies X(2)==myrank.
 */
void FN(bcond_bc)(const orc_params* p, REAL* const a[19])
{
    DECL_SIZES(p);
    const int front = p->bc[ORC_FRONT], rear = p->bc[ORC_REAR], right = p->bc[ORC_RIGHT];
    const int left = p->bc[ORC_LEFT], up = p->bc[ORC_UP], down = p->bc[ORC_DOWN];
    const REAL force = (REAL)((REAL)p->u00 / (REAL)6.0); /* :50-56 */
    const REAL u_inflow = (REAL)p->u_inflow;

    /* ---- front wall (x = l+1) ---- */
    if (front == 0) { /* periodic, :75-105 */
        for (int k = 1; k <= n; ++k) {
            A(12, l1, 0, k) = A(12, 1, m, k); /* SERIAL corner line, :87-92 */
            for (int j = 1; j <= m; ++j) {
                A(10, l1, j, k) = A(10, 1, j, k);
                A(11, l1, j, k) = A(11, 1, j, k);
                A(12, l1, j, k) = A(12, 1, j, k);
                A(13, l1, j, k) = A(13, 1, j, k);
                A(14, l1, j, k) = A(14, 1, j, k);
            }
        }
    }
    if (front == 1) { /* no-slip, :108-124 */
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j) {
                A(12, l1, j - 1, k) = A(1, l, j, k);
                A(13, l1, j, k - 1) = A(2, l, j, k);
                A(10, l1, j + 1, k) = A(3, l, j, k);
                A(11, l1, j, k + 1) = A(4, l, j, k);
                A(14, l1, j, k) = A(5, l, j, k);
            }
    }
    if (front == 5) { /* outflow, :127-205 */
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j) {
                const REAL xj = A(1, l, j, k) + A(2, l, j, k) + A(3, l, j, k) + A(4, l, j, k) +
                                A(5, l, j, k) - A(10, l, j, k) - A(11, l, j, k) - A(12, l, j, k) -
                                A(13, l, j, k) - A(14, l, j, k);
                const REAL yj = A(3, l, j, k) + A(7, l, j, k) + A(8, l, j, k) + A(9, l, j, k) +
                                A(12, l, j, k) - A(1, l, j, k) - A(10, l, j, k) - A(16, l, j, k) -
                                A(17, l, j, k) - A(18, l, j, k);
                const REAL zj = A(4, l, j, k) + A(6, l, j, k) + A(7, l, j, k) + A(13, l, j, k) +
                                A(18, l, j, k) - A(2, l, j, k) - A(9, l, j, k) - A(11, l, j, k) -
                                A(15, l, j, k) - A(16, l, j, k);
                const REAL cvsq = xj * xj + yj * yj + zj * zj;
                const REAL cx10 = RF * (-xj - yj) + QF * ((REAL)3.0 * (xj + yj) * (xj + yj) - cvsq);
                const REAL cx11 = RF * (-xj - zj) + QF * ((REAL)3.0 * (xj + zj) * (xj + zj) - cvsq);
                const REAL cx12 = RF * (-xj + yj) + QF * ((REAL)3.0 * (xj - yj) * (xj - yj) - cvsq);
                const REAL cx13 = RF * (-xj + zj) + QF * ((REAL)3.0 * (xj - zj) * (xj - zj) - cvsq);
                const REAL cx14 = RF * (-xj) + QF * ((REAL)3.0 * (xj) * (xj) - cvsq);
                A(10, l1, j, k) = P2 * ((REAL)1.0 + cx10);
                A(11, l1, j, k) = P2 * ((REAL)1.0 + cx11);
                A(12, l1, j, k) = P2 * ((REAL)1.0 + cx12);
                A(13, l1, j, k) = P2 * ((REAL)1.0 + cx13);
                A(14, l1, j, k) = P1 * ((REAL)1.0 + cx14);
            }
        for (int j = 1; j <= m; ++j) { /* border fix, :172-186 */
            for (int q = 10; q <= 14; ++q) A(q, l1, j, 0) = A(q, l1, j, 1);
            for (int q = 10; q <= 14; ++q) A(q, l1, j, n1) = A(q, l1, j, n);
        }
        for (int k = 1; k <= n; ++k) { /* :189-203 */
            for (int q = 10; q <= 14; ++q) A(q, l1, 0, k) = A(q, l1, 1, k);
            for (int q = 10; q <= 14; ++q) A(q, l1, m1, k) = A(q, l1, m, k);
        }
    }

    /* ---- rear wall (x = 0) ---- */
    if (rear == 0) { /* periodic, :210-238 */
        for (int k = 1; k <= n; ++k) {
            A(1, 0, m1, k) = A(1, l, 1, k); /* SERIAL corner line, :221-225 */
            for (int j = 1; j <= m; ++j) {
                A(1, 0, j, k) = A(1, l, j, k);
                A(2, 0, j, k) = A(2, l, j, k);
                A(3, 0, j, k) = A(3, l, j, k);
                A(4, 0, j, k) = A(4, l, j, k);
                A(5, 0, j, k) = A(5, l, j, k);
            }
        }
    }
    if (rear == 1) { /* no-slip, :241-257 */
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j) {
                A(3, 0, j - 1, k) = A(10, 1, j, k);
                A(4, 0, j, k - 1) = A(11, 1, j, k);
                A(1, 0, j + 1, k) = A(12, 1, j, k);
                A(2, 0, j, k + 1) = A(13, 1, j, k);
                A(5, 0, j, k) = A(14, 1, j, k);
            }
    }
    if (rear == 4) { /* inflow, uniform profile, :260-321 */
        const REAL xj = u_inflow, yj = (REAL)0.0, zj = (REAL)0.0;
        const REAL cvsq = xj * xj + yj * yj + zj * zj;
        const REAL cx01 = RF * (xj - yj) + QF * ((REAL)3.0 * (xj - yj) * (xj - yj) - cvsq);
        const REAL cx02 = RF * (xj - zj) + QF * ((REAL)3.0 * (xj - zj) * (xj - zj) - cvsq);
        const REAL cx03 = RF * (xj + yj) + QF * ((REAL)3.0 * (xj + yj) * (xj + yj) - cvsq);
        const REAL cx04 = RF * (xj + zj) + QF * ((REAL)3.0 * (xj + zj) * (xj + zj) - cvsq);
        const REAL cx05 = RF * (xj) + QF * ((REAL)3.0 * (xj) * (xj) - cvsq);
        for (int k = 0; k <= n1; ++k)
            for (int j = 0; j <= m1; ++j) {
                A(1, 0, j, k) = P2 * ((REAL)1.0 + cx01);
                A(2, 0, j, k) = P2 * ((REAL)1.0 + cx02);
                A(3, 0, j, k) = P2 * ((REAL)1.0 + cx03);
                A(4, 0, j, k) = P2 * ((REAL)1.0 + cx04);
                A(5, 0, j, k) = P1 * ((REAL)1.0 + cx05);
            }
    }

    /* ---- up wall (z = n+1) ---- */
    if (up == 0) { /* periodic, :385-409 */
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                A(2, i, j, n1) = A(2, i, j, 1);
                A(9, i, j, n1) = A(9, i, j, 1);
                A(11, i, j, n1) = A(11, i, j, 1);
                A(15, i, j, n1) = A(15, i, j, 1);
                A(16, i, j, n1) = A(16, i, j, 1);
            }
    }
    if (up == 1 || up == 2) { /* no-slip :412-428, lid :431-447 */
        const REAL f = (up == 2) ? force : (REAL)0.0;
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                A(15, i, j, n1) = A(6, i, j, n);
                A(2, i - 1, j, n1) = (up == 2) ? A(13, i, j, n) + f : A(13, i, j, n);
                A(9, i, j - 1, n1) = A(18, i, j, n);
                A(11, i + 1, j, n1) = (up == 2) ? A(4, i, j, n) - f : A(4, i, j, n);
                A(16, i, j + 1, n1) = A(7, i, j, n);
            }
    }
    if (up == 3) { /* free-slip over the full plane, :450-468 */
        for (int j = 0; j <= m1; ++j)
            for (int i = 0; i <= l1; ++i) {
                A(15, i, j, n1) = A(6, i, j, n);
                A(11, i, j, n1) = A(13, i, j, n);
                A(16, i, j, n1) = A(18, i, j, n);
                A(2, i, j, n1) = A(4, i, j, n);
                A(9, i, j, n1) = A(7, i, j, n);
            }
    }

    /* ---- down wall (z = 0) ---- */
    if (down == 0) { /* periodic, :472-496 */
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                A(4, i, j, 0) = A(4, i, j, n);
                A(6, i, j, 0) = A(6, i, j, n);
                A(7, i, j, 0) = A(7, i, j, n);
                A(13, i, j, 0) = A(13, i, j, n);
                A(18, i, j, 0) = A(18, i, j, n);
            }
    }
    if (down == 1) { /* no-slip, :499-515 */
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                A(6, i, j, 0) = A(15, i, j, 1);
                A(4, i - 1, j, 0) = A(11, i, j, 1);
                A(7, i, j - 1, 0) = A(16, i, j, 1);
                A(13, i + 1, j, 0) = A(2, i, j, 1);
                A(18, i, j + 1, 0) = A(9, i, j, 1);
            }
    }
    if (down == 3) { /* free-slip, interior range only, :518-530 */
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                A(6, i, j, 0) = A(15, i, j, 1);
                A(13, i, j, 0) = A(11, i, j, 1);
                A(18, i, j, 0) = A(16, i, j, 1);
                A(4, i, j, 0) = A(2, i, j, 1);
                A(7, i, j, 0) = A(9, i, j, 1);
            }
    }

    /* ---- left wall (y = 0) ---- */
    if (left == 0) { /* periodic, :535-560 */
        for (int k = 1; k <= n; ++k) {
            A(3, 0, 0, k) = A(3, l, m, k);
            for (int i = 1; i <= l; ++i) {
                A(3, i, 0, k) = A(3, i, m, k);
                A(7, i, 0, k) = A(7, i, m, k);
                A(8, i, 0, k) = A(8, i, m, k);
                A(9, i, 0, k) = A(9, i, m, k);
                A(12, i, 0, k) = A(12, i, m, k);
            }
        }
    }
    if (left == 1) { /* no-slip, :563-579 */
        for (int k = 1; k <= n; ++k)
            for (int i = 1; i <= l; ++i) {
                A(8, i, 0, k) = A(17, i, 1, k);
                A(12, i + 1, 0, k) = A(1, i, 1, k);
                A(3, i - 1, 0, k) = A(10, i, 1, k);
                A(7, i, 0, k - 1) = A(16, i, 1, k);
                A(9, i, 0, k + 1) = A(18, i, 1, k);
            }
    }
    if (left == 3) { /* free-slip, :582-594 */
        for (int k = 1; k <= n; ++k)
            for (int i = 1; i <= l; ++i) {
                A(8, i, 0, k) = A(17, i, 1, k);
                A(3, i, 0, k) = A(1, i, 1, k);
                A(12, i, 0, k) = A(10, i, 1, k);
                A(9, i, 0, k) = A(16, i, 1, k);
                A(7, i, 0, k) = A(18, i, 1, k);
            }
    }

    /* ---- right wall (y = m+1) ---- */
    if (right == 0) { /* periodic, :600-625 */
        for (int k = 1; k <= n; ++k) {
            A(10, l1, m1, k) = A(10, 1, 1, k);
            for (int i = 1; i <= l; ++i) {
                A(1, i, m1, k) = A(1, i, 1, k);
                A(10, i, m1, k) = A(10, i, 1, k);
                A(16, i, m1, k) = A(16, i, 1, k);
                A(17, i, m1, k) = A(17, i, 1, k);
                A(18, i, m1, k) = A(18, i, 1, k);
            }
        }
    }
    if (right == 1) { /* no-slip, :628-644 */
        for (int k = 1; k <= n; ++k)
            for (int i = 1; i <= l; ++i) {
                A(10, i + 1, m1, k) = A(3, i, m, k);
                A(16, i, m1, k + 1) = A(7, i, m, k);
                A(17, i, m1, k) = A(8, i, m, k);
                A(18, i, m1, k - 1) = A(9, i, m, k);
                A(1, i - 1, m1, k) = A(12, i, m, k);
            }
    }
    if (right == 3) { /* free-slip, :647-659 */
        for (int k = 1; k <= n; ++k)
            for (int i = 1; i <= l; ++i) {
                A(1, i, m1, k) = A(3, i, m, k);
                A(18, i, m1, k) = A(7, i, m, k);
                A(17, i, m1, k) = A(8, i, m, k);
                A(16, i, m1, k) = A(9, i, m, k);
                A(10, i, m1, k) = A(12, i, m, k);
            }
    }

    /* ---- free-slip edge fixes, :663-690 ---- */
    if (left == 3 && up == 3)
        for (int i = 1; i <= l; ++i) A(9, i, 0, n1) = A(18, i, 1, n);
    if (right == 3 && up == 3)
        for (int i = 1; i <= l; ++i) A(16, i, m1, n1) = A(7, i, m, n);
    if (right == 3 && down == 3)
        for (int i = 1; i <= l; ++i) A(18, i, m1, 0) = A(9, i, m, 1);
    if (left == 3 && down == 3)
        for (int i = 1; i <= l; ++i) A(7, i, 0, 0) = A(16, i, 1, 1);
}

/* Streaming b_q(x) = a_q(x - c_q) over the interior, CODE/SRC/movef.F90:43-68. */
void FN(movef)(const orc_params* p, REAL* const a[19], REAL* const b[19])
{
    DECL_SIZES(p);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                B(1, i, j, k) = A(1, i - 1, j + 1, k);
                B(2, i, j, k) = A(2, i - 1, j, k + 1);
                B(3, i, j, k) = A(3, i - 1, j - 1, k);
                B(4, i, j, k) = A(4, i - 1, j, k - 1);
                B(5, i, j, k) = A(5, i - 1, j, k);
                B(6, i, j, k) = A(6, i, j, k - 1);
                B(7, i, j, k) = A(7, i, j - 1, k - 1);
                B(8, i, j, k) = A(8, i, j - 1, k);
                B(9, i, j, k) = A(9, i, j - 1, k + 1);
                B(10, i, j, k) = A(10, i + 1, j + 1, k);
                B(11, i, j, k) = A(11, i + 1, j, k + 1);
                B(12, i, j, k) = A(12, i + 1, j - 1, k);
                B(13, i, j, k) = A(13, i + 1, j, k - 1);
                B(14, i, j, k) = A(14, i + 1, j, k);
                B(15, i, j, k) = A(15, i, j, k + 1);
                B(16, i, j, k) = A(16, i, j + 1, k + 1);
                B(17, i, j, k) = A(17, i, j + 1, k);
                B(18, i, j, k) = A(18, i, j + 1, k - 1);
            }
}

/* BGK collision in place on a, reading b01..b18 and a19, all interior nodes
 * including solid ones, CODE/SRC/col.F90:96-235 (FORCING_X default). */
void FN(col)(const orc_params* p, REAL* const a[19], REAL* const b[19])
{
    DECL_SIZES(p);
    REAL omega, fgrad;
    FN(constants)(p, &omega, &fgrad);
    const REAL omega1 = UNO - omega;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const int64_t x = IDX(i, j, k);
                const REAL dx01 = b[0][x], dx02 = b[1][x], dx03 = b[2][x], dx04 = b[3][x];
                const REAL dx05 = b[4][x], dx06 = b[5][x], dx07 = b[6][x], dx08 = b[7][x];
                const REAL dx09 = b[8][x], dx10 = b[9][x], dx11 = b[10][x], dx12 = b[11][x];
                const REAL dx13 = b[12][x], dx14 = b[13][x], dx15 = b[14][x], dx16 = b[15][x];
                const REAL dx17 = b[16][x], dx18 = b[17][x], dx19 = a[18][x];

                const REAL drho = dx01 + dx02 + dx03 + dx04 + dx05 + dx06 + dx07 + dx08 + dx09 +
                                  dx10 + dx11 + dx12 + dx13 + dx14 + dx15 + dx16 + dx17 + dx18 +
                                  dx19;
                const REAL drhoinv = UNO / drho;
                REAL dvx = (dx01 + dx02 + dx03 + dx04 + dx05 - dx10 - dx11 - dx12 - dx13 - dx14) * drhoinv;
                REAL dvy = (dx03 + dx07 + dx08 + dx09 + dx12 - dx01 - dx10 - dx16 - dx17 - dx18) * drhoinv;
                REAL dvz = (dx04 + dx06 + dx07 + dx13 + dx18 - dx02 - dx09 - dx11 - dx15 - dx16) * drhoinv;
                const REAL dvx2 = dvx * dvx, dvy2 = dvy * dvy, dvz2 = dvz * dvz;
                const REAL dvsq = dvx2 + dvy2 + dvz2;

                REAL dvxpy = dvx + dvy;
                const REAL dqxpy = UNO + QF * (TRE * dvxpy * dvxpy - dvsq);
                REAL dvxmy = dvx - dvy;
                const REAL dqxmy = UNO + QF * (TRE * dvxmy * dvxmy - dvsq);
                REAL dvxpz = dvx + dvz;
                const REAL dqxpz = UNO + QF * (TRE * dvxpz * dvxpz - dvsq);
                REAL dvxmz = dvx - dvz;
                const REAL dqxmz = UNO + QF * (TRE * dvxmz * dvxmz - dvsq);
                REAL dvypz = dvy + dvz;
                const REAL dqypz = UNO + QF * (TRE * dvypz * dvypz - dvsq);
                REAL dvymz = dvy - dvz;
                const REAL dqymz = UNO + QF * (TRE * dvymz * dvymz - dvsq);
                const REAL dqx = UNO + QF * (TRE * dvx2 - dvsq);
                const REAL dqy = UNO + QF * (TRE * dvy2 - dvsq);
                const REAL dqz = UNO + QF * (TRE * dvz2 - dvsq);
                dvx = RF * dvx;
                dvy = RF * dvy;
                dvz = RF * dvz;
                dvxpy = RF * dvxpy;
                dvxmy = RF * dvxmy;
                dvxpz = RF * dvxpz;
                dvxmz = RF * dvxmz;
                dvypz = RF * dvypz;
                dvymz = RF * dvymz;

                const REAL drp1 = drho * P1;
                const REAL drp2 = drho * P2;
                const REAL forcex = fgrad * drho, forcey = ZERO, forcez = ZERO;

                const REAL de01 = drp2 * (dvxmy + dqxmy);
                const REAL de02 = drp2 * (dvxmz + dqxmz);
                const REAL de03 = drp2 * (dvxpy + dqxpy);
                const REAL de04 = drp2 * (dvxpz + dqxpz);
                const REAL de05 = drp1 * (dvx + dqx);
                const REAL de06 = drp1 * (dvz + dqz);
                const REAL de07 = drp2 * (dvypz + dqypz);
                const REAL de08 = drp1 * (dvy + dqy);
                const REAL de09 = drp2 * (dvymz + dqymz);
                const REAL de10 = drp2 * (-dvxpy + dqxpy);
                const REAL de11 = drp2 * (-dvxpz + dqxpz);
                const REAL de12 = drp2 * (-dvxmy + dqxmy);
                const REAL de13 = drp2 * (-dvxmz + dqxmz);
                const REAL de14 = drp1 * (-dvx + dqx);
                const REAL de15 = drp1 * (-dvz + dqz);
                const REAL de16 = drp2 * (-dvypz + dqypz);
                const REAL de17 = drp1 * (-dvy + dqy);
                const REAL de18 = drp2 * (-dvymz + dqymz);
                const REAL de19 = drho * P0 * (UNO - QF * dvsq);

                a[0][x] = omega1 * dx01 + (omega * de01 + forcex - forcey);
                a[1][x] = omega1 * dx02 + (omega * de02 + forcex - forcez);
                a[2][x] = omega1 * dx03 + (omega * de03 + forcex + forcey);
                a[3][x] = omega1 * dx04 + (omega * de04 + forcex + forcez);
                a[4][x] = omega1 * dx05 + (omega * de05 + forcex);
                a[5][x] = omega1 * dx06 + (omega * de06 + forcez);
                a[6][x] = omega1 * dx07 + (omega * de07 + forcey + forcez);
                a[7][x] = omega1 * dx08 + (omega * de08 + forcey);
                a[8][x] = omega1 * dx09 + (omega * de09 + forcey - forcez);
                a[9][x] = omega1 * dx10 + (omega * de10 - forcex - forcey);
                a[10][x] = omega1 * dx11 + (omega * de11 - forcex - forcez);
                a[11][x] = omega1 * dx12 + (omega * de12 - forcex + forcey);
                a[12][x] = omega1 * dx13 + (omega * de13 - forcex + forcez);
                a[13][x] = omega1 * dx14 + (omega * de14 - forcex);
                a[14][x] = omega1 * dx15 + (omega * de15 - forcez);
                a[15][x] = omega1 * dx16 + (omega * de16 - forcey - forcez);
                a[16][x] = omega1 * dx17 + (omega * de17 - forcey);
                a[17][x] = omega1 * dx18 + (omega * de18 - forcey + forcez);
                a[18][x] = omega1 * dx19 + (omega * de19);
            }
}

/* One time step = boundaries, propagation, collision, CODE/SRC/bgk3d.F90:128-138
 * (boundaries: bcond_obs then bcond_bc, CODE/SRC/boundaries.F90:36-49,235-248 and
 * CODE/SRC/bcond.comm.packed.F90:394). */
int FN(run)(const orc_params* p, REAL* const a[19], REAL* const b[19], const int32_t* obs,
            int32_t nsteps)
{
    for (int32_t t = 0; t < nsteps; ++t) {
        if (obs) FN(bcond_obs)(p, a, obs);
        FN(bcond_bc)(p, a);
        FN(movef)(p, a, b);
        FN(col)(p, a, b);
    }
    return 0;
}

/*
 * Initial state of the synthetic workloads: rho = 1 and
 * u = (u_in + amp*xi_x, amp*xi_y, amp*xi_z) with xi uniform in [-1, 1) from
 * splitmix64(seed + 3*L + c), L the haloed linear index; populations set to
 * the equilibrium of CODE/SRC/init.F90:194-232 with crho = 1, halos included.
 */
/* The equilibrium of CODE/SRC/init.F90:194-232 at rho = 1 and velocity (xj, yj, zj),
 * stored at haloed index L of the 19 arrays. */
static void FN(equilibrium_at)(REAL xj, REAL yj, REAL zj, REAL* const a[19], int64_t L)
{
    const REAL crho = (REAL)1.0;
    const REAL cvsq = xj * xj + yj * yj + zj * zj;
    const REAL T = (REAL)3.0;
    const REAL cx01 = RF * (xj - yj) + QF * (T * (xj - yj) * (xj - yj) - cvsq);
    const REAL cx02 = RF * (xj - zj) + QF * (T * (xj - zj) * (xj - zj) - cvsq);
    const REAL cx03 = RF * (xj + yj) + QF * (T * (xj + yj) * (xj + yj) - cvsq);
    const REAL cx04 = RF * (xj + zj) + QF * (T * (xj + zj) * (xj + zj) - cvsq);
    const REAL cx05 = RF * (xj) + QF * (T * (xj) * (xj) - cvsq);
    const REAL cx06 = RF * (zj) + QF * (T * (zj) * (zj) - cvsq);
    const REAL cx07 = RF * (yj + zj) + QF * (T * (yj + zj) * (yj + zj) - cvsq);
    const REAL cx08 = RF * (yj) + QF * (T * (yj) * (yj) - cvsq);
    const REAL cx09 = RF * (yj - zj) + QF * (T * (yj - zj) * (yj - zj) - cvsq);
    const REAL cx10 = RF * (-xj - yj) + QF * (T * (xj + yj) * (xj + yj) - cvsq);
    const REAL cx11 = RF * (-xj - zj) + QF * (T * (xj + zj) * (xj + zj) - cvsq);
    const REAL cx12 = RF * (-xj + yj) + QF * (T * (xj - yj) * (xj - yj) - cvsq);
    const REAL cx13 = RF * (-xj + zj) + QF * (T * (xj - zj) * (xj - zj) - cvsq);
    const REAL cx14 = RF * (-xj) + QF * (T * (xj) * (xj) - cvsq);
    const REAL cx15 = RF * (-zj) + QF * (T * (zj) * (zj) - cvsq);
    const REAL cx16 = RF * (-yj - zj) + QF * (T * (yj + zj) * (yj + zj) - cvsq);
    const REAL cx17 = RF * (-yj) + QF * (T * (yj) * (yj) - cvsq);
    const REAL cx18 = RF * (-yj + zj) + QF * (T * (yj - zj) * (yj - zj) - cvsq);
    const REAL cx19 = RF * ((REAL)0.0) + QF * (T * ((REAL)0.0) * ((REAL)0.0) - cvsq);
    a[0][L] = crho * P2 * ((REAL)1.0 + cx01);
    a[1][L] = crho * P2 * ((REAL)1.0 + cx02);
    a[2][L] = crho * P2 * ((REAL)1.0 + cx03);
    a[3][L] = crho * P2 * ((REAL)1.0 + cx04);
    a[4][L] = crho * P1 * ((REAL)1.0 + cx05);
    a[5][L] = crho * P1 * ((REAL)1.0 + cx06);
    a[6][L] = crho * P2 * ((REAL)1.0 + cx07);
    a[7][L] = crho * P1 * ((REAL)1.0 + cx08);
    a[8][L] = crho * P2 * ((REAL)1.0 + cx09);
    a[9][L] = crho * P2 * ((REAL)1.0 + cx10);
    a[10][L] = crho * P2 * ((REAL)1.0 + cx11);
    a[11][L] = crho * P2 * ((REAL)1.0 + cx12);
    a[12][L] = crho * P2 * ((REAL)1.0 + cx13);
    a[13][L] = crho * P1 * ((REAL)1.0 + cx14);
    a[14][L] = crho * P1 * ((REAL)1.0 + cx15);
    a[15][L] = crho * P2 * ((REAL)1.0 + cx16);
    a[16][L] = crho * P1 * ((REAL)1.0 + cx17);
    a[17][L] = crho * P2 * ((REAL)1.0 + cx18);
    a[18][L] = crho * P0 * ((REAL)1.0 + cx19);
}

void FN(init_perturbed)(int32_t l_, int32_t m_, int32_t n_, double u_in, double amp,
                        uint64_t seed, REAL* const a[19])
{
    const int64_t L2 = l_ + 2, M2 = m_ + 2, N2 = n_ + 2;
    const int64_t total = L2 * M2 * N2;
#pragma omp parallel for schedule(static)
    for (int64_t L = 0; L < total; ++L) {
        double xi[3];
        for (int c = 0; c < 3; ++c) {
            const uint64_t h = orc_splitmix64(seed + 3u * (uint64_t)L + (uint64_t)c);
            xi[c] = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
        }
        const REAL xj = (REAL)(u_in + amp * xi[0]);
        const REAL yj = (REAL)(amp * xi[1]);
        const REAL zj = (REAL)(amp * xi[2]);
        FN(equilibrium_at)(xj, yj, zj, a, L);
    }
}

/*
 * The initial states of CODE/SRC/init.F90:42-236, init(opt), for a block of l x m x n
 * nodes starting at start[] (mpicoords * size) in a glob[0] x glob[1] x glob[2] lattice.
 * Coordinates, :110-133: the default build forms them in default REAL (single precision,
 * whatever mykind is), x scaled by nn; -DPERIODIC forms (c + start - 0.5_qp)/size in quad
 * precision and rounds it to mykind -- one division of exact operands in REAL gives the
 * same value.  pi (:61) is a default-REAL parameter, and so are the literals 0.1.
 * Options 4 and 5 stop the reference (:174-188); this returns -1 for them.
 */
int FN(init_reference)(int32_t opt, int32_t l_, int32_t m_, int32_t n_, const int32_t glob[3],
                       const int32_t start[3], int32_t periodic, double u0, REAL* const a[19])
{
    if (opt < 0 || opt > 3) return -1;
    const int64_t L2 = l_ + 2, M2 = m_ + 2;
    const int ll = glob[0], nn = glob[2];
    const REAL pi = (REAL)3.141592653589793238462643383279f;
    const REAL u0m = (REAL)u0;  /* u0 held as real(mykind) */
    for (int k = 0; k <= n_ + 1; ++k) {
        REAL z;
        if (periodic) z = ((REAL)(k + start[2]) - (REAL)0.5) / (REAL)nn;
        else z = (REAL)(((float)(k + start[2]) - 0.5f - 0.5f * (float)nn) / (0.5f * (float)nn));
        for (int j = 0; j <= m_ + 1; ++j) {
            for (int i = 0; i <= l_ + 1; ++i) {
                REAL x;
                if (periodic) x = ((REAL)(i + start[0]) - (REAL)0.5) / (REAL)ll;
                else x = (REAL)(((float)(i + start[0]) - 0.5f - 0.5f * (float)ll) / (0.5f * (float)nn));
                REAL xj = (REAL)0.0, yj = (REAL)0.0, zj = (REAL)0.0;
                if (opt == 1) {                                   /* poiseuille, :148-152 */
                    xj = (REAL)0.1f * ((REAL)1 - z * z);
                }
                if (opt == 2) {                                   /* decaying flow, :154-161 */
                    xj = u0m * RSIN((REAL)2 * pi * z);
                }
                if (opt == 3) {                                   /* kida vortices, :163-171 */
                    xj = (REAL)0.1f * RSIN((REAL)2 * pi * x) * RCOS((REAL)2 * pi * z);
                    zj = -((REAL)0.1f * RCOS((REAL)2 * pi * x) * RSIN((REAL)2 * pi * z));
                }
                FN(equilibrium_at)(xj, yj, zj, a, (int64_t)i + L2 * ((int64_t)j + M2 * (int64_t)k));
            }
        }
    }
    return 0;
}

/*
 * Momentum-exchange force on the solid (no reference counterpart; the
 * reference's drag is the control-volume flux of CODE/SRC/flux_X.F90).  For
 * halfway bounce-back: F = sum over fluid nodes y and directions q whose
 * neighbour y + c_q is solid of 2 c_q a_q(y), a the post-collision state.
 * Neighbours across a periodic axis are wrapped; halo nodes of other faces
 * are never solid.  Accumulated in FP64 in k, j, i, q order.
 */
void FN(mem_force)(const orc_params* p, REAL* const a[19], const int32_t* obs, double out[3])
{
    DECL_SIZES(p);
    static const int cx[18] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0};
    static const int cy[18] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1};
    static const int cz[18] = {0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1};
    const int px = (p->bc[ORC_FRONT] == 0 && p->bc[ORC_REAR] == 0);
    const int py = (p->bc[ORC_RIGHT] == 0 && p->bc[ORC_LEFT] == 0);
    const int pz = (p->bc[ORC_UP] == 0 && p->bc[ORC_DOWN] == 0);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                if (OBS(i, j, k) == 1) continue;
                for (int q = 0; q < 18; ++q) {
                    int ni = i + cx[q], nj = j + cy[q], nk = k + cz[q];
                    if (px) ni = ni < 1 ? ni + l : (ni > l ? ni - l : ni);
                    if (py) nj = nj < 1 ? nj + m : (nj > m ? nj - m : nj);
                    if (pz) nk = nk < 1 ? nk + n : (nk > n ? nk - n : nk);
                    if (ni < 1 || ni > l || nj < 1 || nj > m || nk < 1 || nk > n) continue;
                    if (OBS(ni, nj, nk) != 1) continue;
                    const double f = (double)A(q + 1, i, j, k);
                    fx += 2.0 * cx[q] * f;
                    fy += 2.0 * cy[q] * f;
                    fz += 2.0 * cz[q] * f;
                }
            }
    out[0] = fx;
    out[1] = fy;
    out[2] = fz;
}

/* Global sums of CODE/SRC/diagno.F90:67-120 (solid counts as rho=1, u=0),
 * accumulated in FP64: out = {sum rho, sum ux, sum uy, sum uz, sum u^2}. */
void FN(monitor)(const orc_params* p, REAL* const a[19], const int32_t* obs, double out[5])
{
    DECL_SIZES(p);
    double rt = 0, xt = 0, yt = 0, zt = 0, st = 0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                double rho, xj, yj, zj;
                if (obs && OBS(i, j, k) == 1) {
                    rho = 1.0; xj = yj = zj = 0.0;
                } else {
                    const int64_t x = IDX(i, j, k);
                    double f[19];
                    for (int q = 0; q < 19; ++q) f[q] = (double)a[q][x];
                    rho = 0.0;
                    for (int q = 0; q < 19; ++q) rho += f[q];
                    const double ri = 1.0 / rho;
                    xj = (f[0] + f[1] + f[2] + f[3] + f[4] - f[9] - f[10] - f[11] - f[12] - f[13]) * ri;
                    yj = (f[2] + f[6] + f[7] + f[8] + f[11] - f[0] - f[9] - f[15] - f[16] - f[17]) * ri;
                    zj = (f[3] + f[5] + f[6] + f[12] + f[17] - f[1] - f[8] - f[10] - f[14] - f[15]) * ri;
                }
                rt += rho; xt += xj; yt += yj; zt += zj; st += xj * xj + yj * yj + zj * zj;
            }
    out[0] = rt; out[1] = xt; out[2] = yt; out[3] = zt; out[4] = st;
}

/* Density and velocity per interior node in FP64, interior order (i fastest),
 * as the probe of CODE/SRC/probe_global.F90:58-77 computes them. */
void FN(macro)(const orc_params* p, REAL* const a[19], double* rho, double* ux, double* uy,
               double* uz)
{
    DECL_SIZES(p);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const int64_t x = IDX(i, j, k);
                const int64_t o = (int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1));
                double f[19];
                for (int q = 0; q < 19; ++q) f[q] = (double)a[q][x];
                double r = 0.0;
                for (int q = 0; q < 19; ++q) r += f[q];
                rho[o] = r;
                ux[o] = (f[0] + f[1] + f[2] + f[3] + f[4] - f[9] - f[10] - f[11] - f[12] - f[13]) / r;
                uy[o] = (f[2] + f[6] + f[7] + f[8] + f[11] - f[0] - f[9] - f[15] - f[16] - f[17]) / r;
                uz[o] = (f[3] + f[5] + f[6] + f[12] + f[17] - f[1] - f[8] - f[10] - f[14] - f[15]) / r;
            }
}

/* Macroscopic values of one node in REAL, in the expression order of
 * CODE/SRC/prof_i.F90:45-79 (and varm.F90:53-85): den = a01+...+a19, momentum
 * sums as written there; velocity = momentum/den (div != 0) or
 * momentum*(1/den) (div == 0, varm's rhoinv). */
static void CAT(ref_macro_, P, )(REAL* const a[19], int64_t x, int div, REAL* den, REAL* u, REAL* w, REAL* v)
{
    const REAL r = a[0][x] + a[1][x] + a[2][x] + a[3][x] + a[4][x] + a[5][x] + a[6][x] + a[7][x] + a[8][x] +
                   a[9][x] + a[10][x] + a[11][x] + a[12][x] + a[13][x] + a[14][x] + a[15][x] + a[16][x] +
                   a[17][x] + a[18][x];
    const REAL mx = a[0][x] + a[1][x] + a[2][x] + a[3][x] + a[4][x] - a[9][x] - a[10][x] - a[11][x] - a[12][x] - a[13][x];
    const REAL my = a[2][x] + a[6][x] + a[7][x] + a[8][x] + a[11][x] - a[0][x] - a[9][x] - a[15][x] - a[16][x] - a[17][x];
    const REAL mz = a[3][x] + a[5][x] + a[6][x] + a[12][x] + a[17][x] - a[1][x] - a[8][x] - a[10][x] - a[14][x] - a[15][x];
    *den = r;
    if (div) {
        *u = mx / r; *w = my / r; *v = mz / r;
    } else {
        const REAL ri = UNO / r;
        *u = mx * ri; *w = my * ri; *v = mz * ri;
    }
}

/* Line profile of CODE/SRC/prof_i.F90 (axis 0, at j = c1, k = c2),
 * prof_j.F90 (axis 1, i = c1, k = c2), prof_k.F90 (axis 2, i = c1, j = c2):
 * out[4t + 0..3] = u, w (y), v (z), den of the t-th node, computed in REAL. */
void FN(line)(const orc_params* p, REAL* const a[19], int32_t axis, int32_t c1, int32_t c2, double* out)
{
    DECL_SIZES(p);
    const int len = axis == 0 ? l : (axis == 1 ? m : n);
    for (int t = 1; t <= len; ++t) {
        const int i = axis == 0 ? t : c1, j = axis == 1 ? t : (axis == 0 ? c1 : c2), k = axis == 2 ? t : c2;
        REAL den, u, w, v;
        CAT(ref_macro_, P, )(a, IDX(i, j, k), 1, &den, &u, &w, &v);
        out[4 * (t - 1) + 0] = u; out[4 * (t - 1) + 1] = w; out[4 * (t - 1) + 2] = v; out[4 * (t - 1) + 3] = den;
    }
}

/* Plane means of CODE/SRC/varm.F90:42-98 generalised to any axis: for every
 * plane normal to `axis`, the mean over its nodes of u, w, v (momentum times
 * 1/den in REAL) and den, accumulated in FP64 (the reference accumulates in
 * mykind).  out[4p + 0..3]. */
void FN(plane_means)(const orc_params* p, REAL* const a[19], int32_t axis, double* out)
{
    DECL_SIZES(p);
    const int len = axis == 0 ? l : (axis == 1 ? m : n);
    for (int q = 0; q < 4 * len; ++q) out[q] = 0.0;
    for (int k = 1; k <= n; ++k)
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const int pl = (axis == 0 ? i : (axis == 1 ? j : k)) - 1;
                REAL den, u, w, v;
                CAT(ref_macro_, P, )(a, IDX(i, j, k), 0, &den, &u, &w, &v);
                out[4 * pl + 0] += u; out[4 * pl + 1] += w; out[4 * pl + 2] += v; out[4 * pl + 3] += den;
            }
    const double cnt = axis == 0 ? (double)m * n : (axis == 1 ? (double)l * n : (double)l * m);
    for (int q = 0; q < 4 * len; ++q) out[q] /= cnt;
}

/* Non-equilibrium stress of one node, CODE/SRC/flux_X.F90:162-240 (xx) and
 * CODE/SRC/flux_Y.F90 (xy), in REAL and the reference's expression order. */
static void CAT(ref_stress_, P, )(REAL* const a[19], int64_t x, REAL omega, REAL* sxx, REAL* sxy)
{
    static const int cxl[18] = {1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0};
    static const int cyl[18] = {-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1};
    REAL f[19];
    for (int q = 0; q < 19; ++q) f[q] = a[q][x];
    const REAL rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] +
                     f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    const REAL rhoinv = UNO / rho;
    const REAL xj = (f[0] + f[1] + f[2] + f[3] + f[4] - f[9] - f[10] - f[11] - f[12] - f[13]) * rhoinv;
    const REAL yj = (f[2] + f[6] + f[7] + f[8] + f[11] - f[0] - f[9] - f[15] - f[16] - f[17]) * rhoinv;
    const REAL zj = (f[3] + f[5] + f[6] + f[12] + f[17] - f[1] - f[8] - f[10] - f[14] - f[15]) * rhoinv;
    const REAL cvsq = xj * xj + yj * yj + zj * zj;
    /* rho*w*(1 + rf*e + qf*(3*s*s - cvsq)) with e the signed and s the squared combination */
#define FE(w, e, s) (rho * (w) * (UNO + RF * (e) + QF * (TRE * (s) * (s) - cvsq)))
    REAL fe[18];
    fe[0] = FE(P2, xj - yj, xj - yj);
    fe[1] = FE(P2, xj - zj, xj - zj);
    fe[2] = FE(P2, xj + yj, xj + yj);
    fe[3] = FE(P2, xj + zj, xj + zj);
    fe[4] = FE(P1, xj, xj);
    fe[5] = FE(P1, zj, zj);
    fe[6] = FE(P2, yj + zj, yj + zj);
    fe[7] = FE(P1, yj, yj);
    fe[8] = FE(P2, yj - zj, yj - zj);
    fe[9] = FE(P2, -xj - yj, xj + yj);
    fe[10] = FE(P2, -xj - zj, xj + zj);
    fe[11] = FE(P2, -xj + yj, xj - yj);
    fe[12] = FE(P2, -xj + zj, xj - zj);
    fe[13] = FE(P1, -xj, xj);
    fe[14] = FE(P1, -zj, zj);
    fe[15] = FE(P2, -yj - zj, yj + zj);
    fe[16] = FE(P1, -yj, yj);
    fe[17] = FE(P2, -yj + zj, yj - zj);
#undef FE
    const REAL visc = UNO - (REAL)0.5 * omega;
    REAL xx = -rho / RF, xy = ZERO;
    for (int q = 0; q < 18; ++q) {
        const REAL fn = f[q] - fe[q];
        xx = xx - visc * (REAL)cxl[q] * (REAL)cxl[q] * fn;
        xy = xy - visc * (REAL)cxl[q] * (REAL)cyl[q] * fn;
    }
    *sxx = xx;
    *sxy = xy;
}

/* Control-volume drag of CODE/SRC/drag.F90:51-67 through flux_X.F90 and
 * flux_Y.F90 (serial: offsets 0) for the box box[6] = {xstart, xstop, ystart,
 * ystop, zstart, zstop}: the stresses summed in FP64 over the box faces
 * (the reference sums in mykind).  out = {fluxX, fluxY}. */
void FN(cv_drag)(const orc_params* p, REAL* const a[19], const int32_t box[6], double out[2])
{
    DECL_SIZES(p);
    REAL omega, fgrad;
    FN(constants)(p, &omega, &fgrad);
    int lo[3], hi[3], nrm[3][2], ok[3];
    const int ext[3] = {l, m, n};
    for (int d = 0; d < 3; ++d) {
        const int s0 = box[2 * d], s1 = box[2 * d + 1];
        nrm[d][0] = nrm[d][1] = 1;
        ok[d] = 1;
        if (s0 > 0 && s1 <= ext[d]) { lo[d] = s0; hi[d] = s1; }
        else if (s0 > 0 && s1 > ext[d]) { lo[d] = s0; hi[d] = ext[d]; nrm[d][1] = 0; }
        else if (s0 <= 0 && s1 <= ext[d]) { lo[d] = 1; hi[d] = s1; nrm[d][0] = 0; }
        else ok[d] = 0;
        if (s0 > ext[d] || s1 < 0) ok[d] = 0;
    }
    out[0] = out[1] = 0.0;
    if (!(ok[0] && ok[1] && ok[2])) return;
    double fx[2] = {0.0, 0.0}, fy[2] = {0.0, 0.0};
    for (int f = 0; f < 2; ++f) {
        const int i0 = f ? hi[0] : lo[0];
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j) {
                REAL xx, xy;
                CAT(ref_stress_, P, )(a, IDX(i0, j, k), omega, &xx, &xy);
                fx[f] += xx;
            }
        const int j0 = f ? hi[1] : lo[1];
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                REAL xx, xy;
                CAT(ref_stress_, P, )(a, IDX(i, j0, k), omega, &xx, &xy);
                fy[f] += xy;
            }
    }
    out[0] = -fx[0] * nrm[0][0] + fx[1] * nrm[0][1];
    out[1] = fy[0] * nrm[1][0] + fy[1] * nrm[1][1];
}

#undef RF
#undef QF
#undef UNO
#undef TRE
#undef ZERO
#undef P0
#undef P1
#undef P2
#undef FN
#undef CAT
#undef CAT_

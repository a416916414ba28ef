"""Known-answer tests of the CPU oracle (the reference restatement).

The reference ships no tests or golden vectors, so the oracle is pinned by
analytic properties of the reference's own formulas: the equilibrium of
CODE/SRC/init.F90 has the prescribed moments, equilibrium states are fixed
points of CODE/SRC/col.F90, closed boxes conserve mass, and the halfway
bounce-back of CODE/SRC/bcond.obs.F90 returns a population to the node it left.
"""
import numpy as np
import pytest

from conftest import fluid_mask_haloed

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0])
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0])
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0])
W = np.array([1 / 36] * 4 + [1 / 18] * 2 + [1 / 36, 1 / 18, 1 / 36] + [1 / 36] * 4 + [1 / 18] * 2
             + [1 / 36, 1 / 18, 1 / 36, 1 / 3])


def feq64(rho, u):
    cu = CX * u[0] + CY * u[1] + CZ * u[2]
    usq = u[0] ** 2 + u[1] ** 2 + u[2] ** 2
    return rho * W * (1 + 3 * cu + 4.5 * cu ** 2 - 1.5 * usq)


def test_velocity_table_and_weights():
    # D3Q19: weights sum to one, first moments vanish, second moment is c_s^2 = 1/3
    assert abs(W.sum() - 1) < 1e-15
    for c in (CX, CY, CZ):
        assert abs((W * c).sum()) < 1e-15
        assert abs((W * c * c).sum() - 1 / 3) < 1e-15
    assert (W * CX * CY).sum() == 0


def test_equilibrium_moments(orc):
    a = orc.init_perturbed(6, 5, 4, 0.05, 1e-2, 99, np.float64)
    f = a[:, 2, 2, 3]
    rho = f.sum()
    u = np.array([(f * CX).sum(), (f * CY).sum(), (f * CZ).sum()]) / rho
    assert abs(rho - 1) < 1e-14
    np.testing.assert_allclose(f, feq64(1.0, u), rtol=0, atol=1e-15)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rest_state_is_fixed_point(orc, dtype):
    l, m, n = 10, 8, 6
    p = orc.params(l, m, n, [1, 1, 1, 1, 1, 1], svisc=0.02)
    a = orc.init_perturbed(l, m, n, 0.0, 0.0, 1, dtype)
    a0 = a.copy()
    orc.run(p, a, None, 10)
    tol = 1e-6 if dtype == np.float32 else 1e-15  # a few float ulps per step
    np.testing.assert_allclose(a[:, 1:-1, 1:-1, 1:-1], a0[:, 1:-1, 1:-1, 1:-1], rtol=0, atol=tol)


def test_uniform_flow_invariant_periodic(orc):
    l, m, n = 10, 8, 6
    p = orc.params(l, m, n, [0, 0, 0, 0, 0, 0], svisc=0.02)
    a = orc.init_perturbed(l, m, n, 0.05, 0.0, 1, np.float64)
    a0 = a.copy()
    orc.run(p, a, None, 20)
    np.testing.assert_allclose(a[:, 1:-1, 1:-1, 1:-1], a0[:, 1:-1, 1:-1, 1:-1], rtol=0, atol=1e-15)


def test_single_node_collision_matches_bgk(orc):
    # one interior node of a fully periodic lattice with a non-equilibrium state
    l = m = n = 3
    p = orc.params(l, m, n, [0] * 6, svisc=0.05)
    rng = np.random.default_rng(3)
    b = np.zeros((19, n + 2, m + 2, l + 2))
    a = np.zeros_like(b)
    f = feq64(1.01, np.array([0.03, -0.02, 0.01])) * (1 + 0.05 * rng.standard_normal(19))
    b[:, 2, 2, 2] = f
    a[18, 2, 2, 2] = f[18]
    for q in range(19):
        b[q, 1:-1, 1:-1, 1:-1][b[q, 1:-1, 1:-1, 1:-1] == 0] = W[q]
        a[18][a[18] == 0] = W[18]
    orc.col(p, a, b)
    omega = 2 / (6 * 0.05 + 1)
    rho = f.sum()
    u = np.array([(f * CX).sum(), (f * CY).sum(), (f * CZ).sum()]) / rho
    expect = (1 - omega) * f + omega * feq64(rho, u)
    np.testing.assert_allclose(a[:, 2, 2, 2], expect, rtol=0, atol=1e-15)


@pytest.mark.parametrize("bc", [[1, 1, 1, 1, 1, 1], [1, 1, 1, 1, 0, 0], [1, 1, 0, 0, 1, 1]])
def test_mass_conserved_closed_box(orc, bc):
    l, m, n = 12, 10, 8
    p = orc.params(l, m, n, bc, svisc=0.01)
    a = orc.init_perturbed(l, m, n, 0.02, 1e-2, 7, np.float64)
    obs = np.zeros((n, m, l), np.int32)
    obs[2:5, 3:6, 4:7] = 1
    m0 = orc.monitor(p, a, obs)[0]
    orc.run(p, a, obs, 50)
    assert abs(orc.monitor(p, a, obs)[0] - m0) < 1e-10


def test_bounce_back_returns_population(orc):
    # a single solid voxel: after one step, the fluid neighbour x + c_q receives
    # its own pre-step population heading into the voxel (halfway bounce-back)
    l = m = n = 7
    p = orc.params(l, m, n, [1] * 6, svisc=0.1)
    a = orc.init_perturbed(l, m, n, 0.0, 0.0, 1, np.float64)
    rng = np.random.default_rng(5)
    a[:, 1:-1, 1:-1, 1:-1] *= 1 + 0.1 * rng.random((19, n, m, l))
    obs = np.zeros((n, m, l), np.int32)
    obs[3, 3, 3] = 1  # node (4,4,4)
    pre = a.copy()
    b = np.zeros_like(a)
    orc.bcond_obs(p, a, obs)
    orc.bcond_bc(p, a)
    orc.movef(p, a, b)
    OPP = [11, 12, 9, 10, 13, 14, 15, 16, 17, 2, 3, 0, 1, 4, 5, 6, 7, 8, 18]
    for q in range(18):
        y = (4 + CX[q], 4 + CY[q], 4 + CZ[q])  # fluid node pulling q from the solid voxel
        assert b[q, y[2], y[1], y[0]] == pre[OPP[q], y[2], y[1], y[0]]


def test_links_and_boundary_solid_definitions(orc):
    l, m, n = 9, 8, 7
    p = orc.params(l, m, n, [5, 4, 3, 3, 0, 0], svisc=0.01)
    obs = np.zeros((n, m, l), np.int32)
    obs[:, 2:6, 3:6] = 1  # block spanning z (touches the periodic faces)
    lk = orc.links(p, obs)
    assert np.all((lk[obs == 1] & 0x80000000) != 0)
    # count links directly
    cnt = 0
    for k in range(n):
        for j in range(m):
            for i in range(l):
                if obs[k, j, i]:
                    continue
                for q in range(18):
                    ii, jj, kk = i - CX[q], j - CY[q], k - CZ[q]
                    if 0 <= ii < l and 0 <= jj < m and 0 <= kk < n and obs[kk, jj, ii]:
                        cnt += 1
    assert sum(bin(int(w) & 0x3FFFF).count("1") for w in lk.ravel()) == cnt
    bs = orc.boundary_solid(p, obs)
    # solid voxels with a neighbour that is fluid or halo (halo counts as open)
    expect = []
    for k in range(n):
        for j in range(m):
            for i in range(l):
                if not obs[k, j, i]:
                    continue
                for q in range(18):
                    ii, jj, kk = i + CX[q], j + CY[q], k + CZ[q]
                    if not (0 <= ii < l and 0 <= jj < m and 0 <= kk < n) or not obs[kk, jj, ii]:
                        expect.append(i + l * (j + m * k))
                        break
    assert bs.tolist() == expect
    assert len(bs) == obs.sum() - 10  # the 1x2 core column of the 3x4 block is enclosed for k = 2..6


def test_frozen_edge_ghosts_keep_initial_values(orc):
    # free-slip y + periodic z: the y-z ghost edge lines a07(:,0,0), a09(:,0,n1),
    # a16(:,m1,n1), a18(:,m1,0) are written by no block of CODE/SRC/bcond.bc.F90
    l, m, n = 8, 6, 5
    p = orc.params(l, m, n, [5, 4, 3, 3, 0, 0], svisc=0.01, u_inflow=0.05)
    a = orc.init_perturbed(l, m, n, 0.05, 1e-3, 11)
    a0 = a.copy()
    orc.run(p, a, None, 5)
    for q, j, k in ((6, 0, 0), (8, 0, n + 1), (15, m + 1, n + 1), (17, m + 1, 0)):
        assert np.array_equal(a[q, k, j, 1:-1], a0[q, k, j, 1:-1])
    assert not np.array_equal(a[6, 1, 0, 1:-1], a0[6, 1, 0, 1:-1])  # an ordinary ghost row does change


def test_mem_force_sign_and_symmetry(orc):
    # uniform flow in +x on a y/z-symmetric obstacle: drag along +x, no lift
    l, m, n = 24, 12, 12
    p = orc.params(l, m, n, [5, 4, 1, 1, 1, 1], svisc=0.05, u_inflow=0.05)
    a = orc.init_perturbed(l, m, n, 0.05, 0.0, 1, np.float64)
    obs = np.zeros((n, m, l), np.int32)
    obs[4:8, 4:8, 8:12] = 1
    orc.run(p, a, obs, 30)
    f = orc.mem_force(p, a, obs)
    assert f[0] > 0
    assert abs(f[1]) < 1e-10 * abs(f[0]) + 1e-13 and abs(f[2]) < 1e-10 * abs(f[0]) + 1e-13


def test_halo_mask_helper():
    obs = np.zeros((2, 3, 4), np.int32)
    obs[1, 1, 2] = 1
    k = fluid_mask_haloed(obs)
    assert k.shape == (4, 5, 6) and (~k).sum() == 1 and not k[2, 2, 3]

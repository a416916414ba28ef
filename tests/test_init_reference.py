"""CPU tests of eup_init_reference, the reference's initial states init(opt)
(CODE/SRC/init.F90, options 0..3): equal to the oracle's line-by-line
restatement in both precisions, with both coordinate forms, on whole lattices
and on the blocks of a process grid; the blocks tile the whole lattice; the
fields have the velocities the options describe; options the reference stops
on are refused."""
import numpy as np
import pytest


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("opt", [0, 1, 2, 3])
def test_matches_oracle(eup, orc, dtype, periodic, opt):
    for l, m, n, glob, start in [(20, 12, 10, None, (0, 0, 0)), (10, 6, 5, (20, 12, 10), (10, 6, 5)),
                                 (7, 9, 11, (21, 9, 33), (14, 0, 11))]:
        got = eup.init_reference(opt, l, m, n, glob, start, periodic, 0.05, dtype)
        want = orc.init_reference(opt, l, m, n, glob, start, periodic, 0.05, dtype)
        assert np.array_equal(got, want), (l, m, n, start)


@pytest.mark.parametrize("periodic", [False, True])
def test_blocks_tile_the_lattice(eup, periodic):
    lx, ly, lz = 24, 12, 10
    whole = eup.init_reference(3, lx, ly, lz, periodic=periodic)
    l, m, n = 12, 6, 5
    for s in [(0, 0, 0), (12, 6, 5), (12, 0, 5), (0, 6, 0)]:
        block = eup.init_reference(3, l, m, n, (lx, ly, lz), s, periodic)
        sub = whole[:, s[2]:s[2] + n + 2, s[1]:s[1] + m + 2, s[0]:s[0] + l + 2]
        assert np.array_equal(block, sub), s


def _velocity(a):
    cx = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], float)
    cz = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], float)
    a = a.astype(np.float64)
    rho = a.sum(0)
    return rho, np.tensordot(cx, a, 1) / rho, np.tensordot(cz, a, 1) / rho


def test_fields(eup):
    l, m, n = 16, 4, 20
    rho, ux, uz = _velocity(eup.init_reference(0, l, m, n, dtype=np.float64))
    assert np.allclose(rho, 1, atol=1e-14) and np.abs(ux).max() < 1e-15
    # Poiseuille: u_x = 0.1 (1 - z^2), z = (k - 0.5 - n/2)/(n/2) in (-1, 1)
    rho, ux, uz = _velocity(eup.init_reference(1, l, m, n, dtype=np.float64))
    k = np.arange(n + 2)
    z = (k - 0.5 - 0.5 * n) / (0.5 * n)
    np.testing.assert_allclose(ux[:, 3, 5], 0.1 * (1 - z * z), rtol=1e-6, atol=1e-7)
    # decaying shear: u_x = u0 sin(2 pi z)
    rho, ux, uz = _velocity(eup.init_reference(2, l, m, n, u0=0.04, dtype=np.float64))
    np.testing.assert_allclose(ux[:, 3, 5], 0.04 * np.sin(2 * np.pi * z), rtol=1e-5, atol=1e-7)
    # Kida vortices (periodic coordinates): divergence-free pair, amplitude 0.1
    rho, ux, uz = _velocity(eup.init_reference(3, l, m, n, periodic=True, dtype=np.float64))
    assert abs(np.abs(ux).max() - 0.1) < 0.01 and abs(np.abs(uz).max() - 0.1) < 0.01


def test_refused_options(eup):
    for opt, code in [(4, 5), (5, 5), (6, 1), (-1, 1)]:
        with pytest.raises(eup.EupError) as e:
            eup.init_reference(opt, 8, 8, 8)
        assert e.value.code == code, opt

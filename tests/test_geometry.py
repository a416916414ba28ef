"""CPU tests of the host voxeliser (the node tests it shares with the device
voxeliser): the obstacles the reference creates (CODE/SRC/build.obs.F90,
flag1 = 2) against the oracle's line-by-line restatement, on whole lattices and
on the blocks of a process grid; the synthetic shells' helpers; the obstacle
file layout; and the accuracy of the voxelisers' atan2."""
import ctypes
import math

import numpy as np
import pytest

SIZES = [(96, 64, 48), (130, 70, 66), (256, 128, 64)]


@pytest.mark.parametrize("flag2", [1, 2, 3])
@pytest.mark.parametrize("cylinder_inf,test1", [(False, False), (True, False), (False, True)])
def test_reference_shapes_match_oracle(eup, orc, flag2, cylinder_inf, test1):
    for lx, ly, lz in SIZES:
        g = eup.geometry_reference(flag2, lx, ly, lz, cylinder_inf=cylinder_inf, test1=test1)
        want, nobs = orc.created_obstacle(flag2, lx, ly, lz, lx, ly, lz, cylinder_inf=cylinder_inf, test1=test1)
        got = eup.voxelise(g, lx, ly, lz)
        assert np.array_equal(got, want), (lx, ly, lz)
        assert got.sum() > 0 and nobs == got.sum() - 100  # the reference's counter starts at -100
        # the blocks of a 2x2x2 process grid: offset = mpicoords * local size
        l, m, n = lx // 2, ly // 2, lz // 2
        for c in [(0, 0, 0), (1, 0, 1), (1, 1, 1), (0, 1, 0)]:
            w, _ = orc.created_obstacle(flag2, lx, ly, lz, l, m, n, mpicoords=c, cylinder_inf=cylinder_inf,
                                        test1=test1)
            assert np.array_equal(eup.voxelise(g.shifted((c[0] * l, c[1] * m, c[2] * n)), l, m, n), w), c


def test_reference_shape_parameters(eup):
    g = eup.geometry_reference(2, 400, 200, 40, cylinder_inf=True)
    assert g.kind == eup.GEOM_REF_COLUMN and list(g.center) == [100, 100, 0]
    assert (g.r2_lo, g.r2_hi, g.kstop) == (0, 102 * 102, 41)
    g = eup.geometry_reference(2, 400, 200, 40)  # radius min(20, lx/8), k < lz
    assert (g.r2_hi, g.kstop) == (22 * 22, 40)
    g = eup.geometry_reference(3, 400, 200, 40)  # radius min(20, lz/8), k < 60
    assert (g.r2_hi, g.kstop) == (7 * 7, 60)
    g = eup.geometry_reference(1, 400, 200, 40)
    assert g.kind == eup.GEOM_REF_SPHERE and list(g.center) == [100, 100, 20]
    assert (g.r2_lo, g.r2_hi) == (18 * 18, 22 * 22)
    with pytest.raises(eup.EupError) as e:
        eup.geometry_reference(4, 64, 64, 64)
    assert e.value.code == 5
    with pytest.raises(eup.EupError) as e:  # unknown variant bit
        eup._check(eup.lib.eup_geometry_reference(1, 64, 64, 64, 8, ctypes.byref(eup.Geometry())))
    assert e.value.code == 1


def test_voxelise_rejects_bad_shapes(eup):
    with pytest.raises(eup.EupError):
        eup.voxelise(eup.Geometry(kind=99), 8, 8, 8)
    with pytest.raises(eup.EupError):
        eup.voxelise(eup.Geometry.reticular_shell(4, 8, 4, 4, 2, 3, 1, 0), 8, 8, 8)  # outer_d < strut_d
    with pytest.raises(eup.EupError):
        eup.voxelise(eup.Geometry.ridged_shell(4, 8, 4, 4, 6, 1, 2, 1, 0, 1, 1, 0), 8, 8, 8)  # ridge_t = 0


def test_shell_helpers_are_the_voxeliser(eup):
    l, m, n = 160, 72, 73
    args = (40, 64, 36.5, 37.0, 48, 4, 16)
    obs = eup.geometry_reticular_shell(l, m, n, *args, 7)
    assert np.array_equal(obs, eup.voxelise(eup.Geometry.reticular_shell(*args, 7), l, m, n))
    # the ridged mask is the solid-fraction field at smooth_w = 0, thresholded at 1/2
    ridged = eup.Geometry.ridged_shell(*args, 4.0, 3.0, 4.0, 5.0, 7)
    ns = eup.geometry_ridged_shell(l, m, n, *args, 4.0, 3.0, 4.0, 5.0, 0.0, 7)
    mask = eup.voxelise(ridged, l, m, n)
    assert np.array_equal(mask, (ns >= 0.5).astype(np.int32)) and mask.sum() > obs.sum()
    cyl = eup.voxelise(eup.Geometry.cylinder_z(20.5, 30, 6.5), l, m, n)
    assert np.array_equal(cyl, eup.geometry_cylinder_z(l, m, n, 20.5, 30, 6.5))


@pytest.mark.parametrize("kind", ["reticular", "ridged", "cylinder"])
def test_voxelise_blocks_tile_the_lattice(eup, kind):
    """Offsets place a block in the global lattice: the x-slabs (and any process grid) of a
    shape tile the whole lattice's mask."""
    lx, ly, lz = 150, 64, 60
    args = (30, 80, 32.5, 30.0, 40, 4, 12)
    g = {"reticular": eup.Geometry.reticular_shell(*args, 3),
         "ridged": eup.Geometry.ridged_shell(*args, 4.0, 3.0, 3.0, 5.0, 3),
         "cylinder": eup.Geometry.cylinder_z(70.5, 33, 9)}[kind]
    full = eup.voxelise(g, lx, ly, lz)
    assert full.sum() > 0
    for x0, nx in [(1, 37), (38, 40), (78, 73)]:
        part = eup.voxelise(g.shifted((x0 - 1, 0, 0)), nx, ly, lz)
        assert np.array_equal(part, full[:, :, x0 - 1:x0 - 1 + nx]), x0
    part = eup.voxelise(g.shifted((50, 20, 30)), 60, 30, 30)
    assert np.array_equal(part, full[30:60, 20:50, 50:110])


def test_obstacle_file_layout(eup, orc, tmp_path):
    """eup_write_obs_file writes the oracle's bytes of CODE/SRC/build.obs.F90:506-541."""
    lx, ly, lz = 96, 64, 48
    g = eup.geometry_reference(1, lx, ly, lz)
    obs = eup.voxelise(g, lx, ly, lz)
    path = tmp_path / "obs.0000.00000000.bin"
    eup._check(eup.lib.eup_write_obs_file(str(path).encode(), lx, ly, lz, obs.ctypes.data))
    assert path.read_bytes() == orc.obstacle_file_bytes(obs)
    back, nobs = eup.read_obs_file(str(path), lx, ly, lz)
    assert nobs == obs.sum() and np.array_equal(back, obs)


def test_atan2_det_accuracy(eup):
    """The voxelisers' atan2, from basic operations only, is within 2 ulp of libm's."""
    f = eup.lib.eup_internal_atan2_det
    f.argtypes, f.restype = [ctypes.c_double, ctypes.c_double], ctypes.c_double
    rng = np.random.default_rng(5)
    pts = list(rng.uniform(-300, 300, size=(20000, 2)))
    pts += [(float(a), float(b)) for a in range(-6, 7) for b in range(-6, 7)]
    pts += [(0.5, 0.5), (1e-300, 1.0), (1.0, 1e-300), (-0.0, -1.0), (3.0, -3.0), (-2.5, -2.5)]
    worst = 0.0
    for y, x in pts:
        want = math.atan2(y, x)
        got = f(y, x)
        if want == 0.0:
            assert got == 0.0 or abs(got) < 1e-300
            continue
        worst = max(worst, abs(got - want) / math.ulp(want))
    assert worst <= 2.0, worst
    assert f(0.0, 0.0) == 0.0

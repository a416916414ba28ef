"""The device voxeliser (eup_build_obstacles): its bit-packed mask equals the
host voxeliser's (the same node tests, compiled for both sides) for every shape,
offset and ragged row length; installing it is the same as installing that mask
through eup_set_obstacles (same boundary list, links and time steps, bit for
bit); the obstacle file it writes from the device equals the reference layout
(CODE/SRC/build.obs.F90:506-541); its checks reject what eup_set_obstacles
rejects and keep the previous mask; and the reference program, fed flag1 = 2,
creates the reference's column on the device and steps like the oracle."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "euplectella_hpc_b200", "_lib",
                      "eup_bgk3d")
ALL_PERIODIC = (0, 0, 0, 0, 0, 0)


def shapes(eup):
    """(name, geometry, lattice) cases: every kind, rows not a multiple of 32, offsets."""
    G = eup.Geometry
    return [
        ("sphere", eup.geometry_reference(1, 97, 64, 50), (97, 64, 50)),
        ("sphere_test1", eup.geometry_reference(1, 150, 90, 70, test1=True), (150, 90, 70)),
        ("column", eup.geometry_reference(2, 160, 70, 33), (160, 70, 33)),
        ("column_inf", eup.geometry_reference(2, 250, 232, 12, cylinder_inf=True), (250, 232, 12)),
        ("half_column", eup.geometry_reference(3, 120, 64, 72), (120, 64, 72)),
        ("column_block", eup.geometry_reference(2, 160, 70, 33).shifted((80, 35, 0)), (80, 35, 33)),
        ("cylinder_z", G.cylinder_z(40.5, 31, 9.5), (131, 64, 9)),
        ("reticular", G.reticular_shell(30, 80, 32.5, 30.0, 40, 4, 12, 3), (150, 64, 60)),
        ("reticular_seed", G.reticular_shell(20, 64, 36.0, 36.5, 48, 3, 10, 11), (100, 72, 73)),
        ("reticular_slab", G.reticular_shell(30, 80, 32.5, 30.0, 40, 4, 12, 3).shifted((37, 0, 0)), (41, 64, 60)),
        ("ridged", G.ridged_shell(30, 80, 32.5, 30.0, 40, 4, 12, 4.0, 3.0, 3.0, 5.0, 3), (150, 64, 60)),
        ("none", G(kind=eup.GEOM_NONE), (40, 8, 8)),
    ]


def test_device_mask_equals_host_mask(eup, require_gpu):
    for name, g, (l, m, n) in shapes(eup):
        want = eup.voxelise(g, l, m, n)
        with eup.Solver(eup.Config(l, m, n, bc=ALL_PERIODIC)) as s:
            s.build_obstacles(g)
            got, nobs = s.obstacles()
            assert s.obstacle_count() == nobs
        assert nobs == int(want.sum()), name
        assert np.array_equal(got, want), (name, int((got != want).sum()))


def test_build_equals_set_through_steps(eup, orc, require_gpu):
    """Installing the device-built mask is installing the host mask: same boundary solids,
    links, forces and state after 30 steps, bit for bit (and equal to the oracle)."""
    l, m, n = 96, 48, 16
    g = eup.Geometry.reticular_shell(24, 48, 24.5, 8.5, 14, 3, 6, 5)
    obs = eup.voxelise(g, l, m, n)
    assert obs.sum() > 100
    cfg = eup.Config(l, m, n, bc=(5, 4, 3, 3, 0, 0), svisc=0.02, u_inflow=0.05)
    a0 = eup.init_equilibrium(l, m, n, 0.05, 1e-3, 9, np.float32)
    out = []
    for build in (True, False):
        with eup.Solver(cfg) as s:
            if build:
                s.build_obstacles(g)
            else:
                s.set_obstacles(obs)
            s.upload(a0)
            bs, lk = s.boundary_solid(), s.links()
            s.step(30)
            out.append((bs, lk, s.download(np.float32), s.force_series(0, 31)))
    (bs1, lk1, a1, f1), (bs2, lk2, a2, f2) = out
    assert np.array_equal(bs1, bs2) and np.array_equal(lk1, lk2)
    assert np.array_equal(a1, a2) and np.array_equal(f1, f2)
    p = orc.params(l, m, n, cfg.bc, svisc=0.02, u_inflow=0.05)
    ref = a0.copy()
    orc.run(p, ref, obs, 30)
    keep = np.ones(ref.shape[1:], bool)
    keep[1:-1, 1:-1, 1:-1] = obs == 0
    for q in range(19):
        assert np.array_equal(a1[q][keep], ref[q][keep]), q


def test_write_obstacles_from_the_device(eup, orc, require_gpu, tmp_path):
    for name, g, (l, m, n) in shapes(eup):
        want = eup.voxelise(g, l, m, n)
        path = tmp_path / f"obs.{name}.bin"
        with eup.Solver(eup.Config(l, m, n, bc=ALL_PERIODIC)) as s:
            s.build_obstacles(g)
            s.write_obstacles(path)
        assert path.read_bytes() == orc.obstacle_file_bytes(want), name
        back, nobs = eup.read_obs_file(str(path), l, m, n)
        assert nobs == want.sum() and np.array_equal(back, want), name


def test_build_obstacles_checks_keep_the_previous_mask(eup, require_gpu):
    l, m, n = 64, 32, 8
    inside = eup.Geometry.cylinder_z(20, 16.5, 4)
    with eup.Solver(eup.Config(l, m, n, bc=(5, 4, 3, 3, 0, 0), u_inflow=0.05)) as s:
        s.build_obstacles(inside)
        before, cnt = s.obstacles()
        assert cnt > 0
        for bad, code in [(eup.Geometry.cylinder_z(63, 16.5, 3), 5),    # solid on the outflow plane i = l
                          (eup.Geometry(kind=42), 1),                    # unknown shape
                          (eup.Geometry.reticular_shell(4, 8, 4, 4, 2, 3, 1, 0), 1)]:
            with pytest.raises(eup.EupError) as e:
                s.build_obstacles(bad)
            assert e.value.code == code
            after, c2 = s.obstacles()
            assert c2 == cnt and np.array_equal(after, before)
        s.build_obstacles(eup.Geometry(kind=eup.GEOM_NONE))  # clears the mask
        assert s.obstacle_count() == 0 and not s.obstacles()[0].any()
        s.set_obstacles(before)  # the host path still installs over a device-built one
        assert s.obstacle_count() == cnt
    # an x-slab face: no solid on the column next to it
    with eup.Solver(eup.Config(l, m, n, bc=(eup.EXCHANGE, 4, 3, 3, 0, 0), u_inflow=0.05)) as s:
        with pytest.raises(eup.EupError) as e:
            s.build_obstacles(eup.Geometry.cylinder_z(64, 16.5, 2))
        assert e.value.code == 5
    # a solid-fraction field excludes halfway-bounce-back voxels
    with eup.Solver(eup.Config(l, m, n, bc=(5, 4, 3, 3, 0, 0), u_inflow=0.05)) as s:
        s.set_solid_fraction(np.zeros((n, m, l)))
        with pytest.raises(eup.EupError) as e:
            s.build_obstacles(inside)
        assert e.value.code == 5


def test_slabs_build_their_block(eup, require_gpu):
    """Each x-slab voxelises its own block of the global shape (offset x0 - 1).  The shell
    lies inside the middle slab (columns 81..160): a solid next to an exchange face is
    rejected, as with eup_set_obstacles."""
    from euplectella_hpc_b200.slabs import SlabSolver, slab_obstacles
    cfg = eup.Config(240, 64, 60, bc=(5, 4, 3, 3, 3, 3), u_inflow=0.05)
    g = eup.Geometry.reticular_shell(95, 48, 32.5, 30.0, 40, 4, 12, 3)
    full = eup.voxelise(g, cfg.lx, cfg.ly, cfg.lz)
    assert full[:, :, 92:146].sum() == full.sum() > 0
    for rank in range(3):
        s = SlabSolver(cfg, rank, 3)
        try:
            s.build_obstacles(g)
            assert np.array_equal(s.solver.obstacles()[0], slab_obstacles(full, s.x0, s.nx)), rank
        finally:
            s.solver.close()
    s = SlabSolver(cfg, 1, 2)  # columns 121..240: the face at x = 121 cuts the shell
    try:
        with pytest.raises(eup.EupError) as e:
            s.build_obstacles(g)
        assert e.value.code == 5
    finally:
        s.solver.close()


def test_driver_creates_the_reference_column(eup, orc, require_gpu, tmp_path):
    """flag1 = 2, flag2 = 2 with the FREESLIP preset: the reference's column (radius
    min(20, lx/8), k < lz) built on the device, dumped with flag3 = 2, and stepped."""
    lx, ly, lz = 96, 48, 16
    a = eup.init_equilibrium(lx, ly, lz, 0.05, 1e-3, 23, np.float32)
    eup.write_raw_state(tmp_path / "restore.00.00.00.bin", a, 0)
    (tmp_path / "bgk.input").write_text(
        f"&parameters\n lx = {lx}\n ly = {ly}\n lz = {lz}\n proc_x = 1\n proc_y = 1\n proc_z = 1\n"
        " svisc=0.02\n u0=0.05\n itfin=20\n ivtim=1000\n isignal=20\n itsave=20\n icheck=10\n"
        " tstep=10\n irestart=1\n flag1=2\n flag2=2\n flag3=2\n init_v=0        /\n")
    r = subprocess.run([DRIVER, "--preset", "freeslip"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    obs, nobs = orc.created_obstacle(2, lx, ly, lz, lx, ly, lz)
    assert obs.sum() > 0 and not obs[lz - 1].any()  # the top layer k = lz stays fluid
    assert (tmp_path / "obs.0000.00000000.bin").read_bytes() == orc.obstacle_file_bytes(obs)
    assert f"num. obs       --> {int(obs.sum())}" in r.stdout
    p = orc.params(lx, ly, lz, [5, 4, 3, 3, 3, 3], svisc=0.02, u_inflow=0.05)
    ref = a.copy()
    orc.run(p, ref, obs, 20)
    got, it = eup.read_raw_state(tmp_path / "save.00.00.00.00000020.bin", lx, ly, lz)
    assert it == 20
    keep = np.ones(got.shape[1:], bool)
    keep[1:-1, 1:-1, 1:-1] = obs == 0
    for q in range(19):
        assert np.array_equal(got[q][keep], ref[q][keep]), q


def test_driver_production_column(eup, orc, require_gpu, tmp_path):
    """The obstacle of the reference's production inputs (CODE/RUN/bgk.*.input: flag1 = 2,
    flag2 = 2, built with -DCYLINDER_INF): the radius-100 column over every z layer, created on
    the device by the reference program on a 420x210x4 channel and stepped like the oracle."""
    lx, ly, lz = 420, 210, 4
    a = eup.init_equilibrium(lx, ly, lz, 0.05, 1e-3, 29, np.float32)
    eup.write_raw_state(tmp_path / "restore.00.00.00.bin", a, 0)
    (tmp_path / "bgk.input").write_text(
        f"&parameters\n lx = {lx}\n ly = {ly}\n lz = {lz}\n proc_x = 1\n proc_y = 1\n proc_z = 1\n"
        " svisc=0.02\n u0=0.05\n itfin=10\n ivtim=1000\n isignal=10\n itsave=10\n icheck=10\n"
        " tstep=10\n irestart=1\n flag1=2\n flag2=2\n flag3=2\n init_v=0        /\n")
    r = subprocess.run([DRIVER, "--preset", "cylinder_inf"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    obs, _ = orc.created_obstacle(2, lx, ly, lz, lx, ly, lz, cylinder_inf=True)
    assert obs[-1].sum() == obs[0].sum() > 0 and not obs[:, :, -1].any()  # every layer, clear of i = l
    assert (tmp_path / "obs.0000.00000000.bin").read_bytes() == orc.obstacle_file_bytes(obs)
    p = orc.params(lx, ly, lz, [5, 4, 0, 0, 0, 0], svisc=0.02, u_inflow=0.05)
    ref = a.copy()
    orc.run(p, ref, obs, 10)
    got, it = eup.read_raw_state(tmp_path / "save.00.00.00.00000010.bin", lx, ly, lz)
    assert it == 10
    keep = np.ones(got.shape[1:], bool)
    keep[1:-1, 1:-1, 1:-1] = obs == 0
    for q in range(19):
        assert np.array_equal(got[q][keep], ref[q][keep]), q

"""The eup_bgk3d program: the reference's serial program over the C ABI, fed
the reference's own input files (bgk.input namelist, obs.0000.00000000.bin,
restore.00.00.00.bin).  Its save files must equal the oracle's state bit for
bit and its drag lines the oracle's momentum exchange."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "euplectella_hpc_b200", "_lib",
                      "eup_bgk3d")


def test_driver_runs_reference_inputs(eup, orc, require_gpu, tmp_path):
    l, m, n = 40, 24, 12
    obs = eup.geometry_cylinder_z(l, m, n, 12, 12.5, 3.5)
    eup.write_obs_file(tmp_path / "obs.0000.00000000.bin", obs)
    a = eup.init_equilibrium(l, m, n, 0.05, 1e-3, 17, np.float32)
    eup.write_raw_state(tmp_path / "restore.00.00.00.bin", a, 100)
    (tmp_path / "bgk.input").write_text(
        "&parameters\n lx = 40\n ly = 24\n lz = 12\n proc_x = 1\n proc_y = 1\n proc_z = 1\n"
        " svisc=0.01,0.005\n u0=0.05\n itfin=140\n ivtim=1000\n isignal=20\n itsave=20\n icheck=10\n"
        " tstep=10\n irestart=1\n flag1=1\n flag2=2\n flag3=0\n init_v=0        /\n")
    r = subprocess.run([DRIVER, "--preset", "cylinder_inf", "--drag-length", "7", "--cv-drag"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    # oracle with the CYLINDER_INF flags (in/out x, periodic y and z), u_inflow = u0
    p = orc.params(l, m, n, [5, 4, 0, 0, 0, 0], svisc=0.01, u_inflow=0.05)
    ref = a.copy()
    forces = {}
    for t in range(101, 141):
        orc.run(p, ref, obs, 1)
        if t % 10 == 0:
            forces[t] = orc.mem_force(p, ref, obs)
        if t % 20 == 0:
            got, it = eup.read_raw_state(tmp_path / f"save.00.00.00.{t:08d}.bin", l, m, n)
            assert it == t
            keep = np.ones(got.shape[1:], bool)
            keep[1:-1, 1:-1, 1:-1] = obs == 0
            for q in range(19):
                assert np.array_equal(got[q][keep], ref[q][keep]), (t, q)
    lines = (tmp_path / "drag_mem.0000.dat").read_text().split("\n")
    rows = [list(map(float, ln.split())) for ln in lines if ln.strip()]
    assert [int(r_[0]) for r_ in rows] == [110, 120, 130, 140]
    for row in rows:
        np.testing.assert_allclose(row[1:4], forces[int(row[0])], rtol=1e-12, atol=1e-14)
        assert abs(row[4] - row[1] / (0.5 * 0.05 ** 2 * 7 * n)) <= 1e-12 * abs(row[4])
    # profiles and plane means of the last check (t = 140) against the oracle's final state,
    # to the 6 significant digits of the e14.6 format (half a unit of the 6th digit: 5e-6 relative)
    def last_block(name):
        text = (tmp_path / name).read_text()
        blk = text.split("# t=")[-1].split("\n")
        assert int(blk[0]) == 140
        return np.array([list(map(float, ln.split())) for ln in blk[1:] if ln.strip()])
    for ax, fname, (c1, c2) in ((0, "prof_i.0000.dat", (m // 2, n // 2)), (1, "prof_j.0000.dat", (l // 2, n // 2)),
                                (2, "prof_k.0000.dat", (l // 2, m // 2))):
        rows_ = last_block(fname)
        want = orc.line(p, ref, ax, c1, c2)
        assert rows_.shape == (want.shape[0], 5)
        fluid = [obs[c2 - 1, c1 - 1, :], obs[c2 - 1, :, c1 - 1], obs[:, c2 - 1, c1 - 1]][ax] == 0
        bad = ~np.isclose(rows_[fluid, 1:], want[fluid], rtol=5e-6, atol=1e-12)
        assert not bad.any(), (fname, np.argwhere(bad)[:5].tolist(), rows_[fluid][bad.any(1)][:3].tolist(),
                               want[fluid][bad.any(1)][:3].tolist())
    assert last_block("u_med.000.000.000.dat").shape == (n, 5)
    cv = [ln.split() for ln in (tmp_path / "drag.0000.dat").read_text().split("\n") if ln.strip()]
    assert len(cv) == 4 * 4 and [int(c[0]) for c in cv[:4]] == [52, 57, 62, 67]
    probe = (tmp_path / "probe_g.0000.dat").read_text().split("\n")[0]
    assert probe.startswith("     110") and "E" in probe
    assert "Mlups" in (tmp_path / "bgk.perf").read_text()


@pytest.mark.parametrize("init_v,periodic", [(1, False), (3, True)])
def test_driver_reference_initial_states(eup, orc, require_gpu, tmp_path, init_v, periodic):
    """init_v = 1 (Poiseuille) and 3 (Kida vortices, -DPERIODIC coordinates) built by the
    program through eup_init_reference, stepped on a fully periodic box like the oracle."""
    l, m, n = 32, 12, 16
    (tmp_path / "bgk.input").write_text(
        f"&parameters\n lx = {l}\n ly = {m}\n lz = {n}\n proc_x = 1\n proc_y = 1\n proc_z = 1\n"
        " svisc=0.02\n u0=0.0\n itfin=10\n ivtim=1000\n isignal=10\n itsave=10\n icheck=10\n"
        f" tstep=10\n irestart=0\n flag1=0\n flag2=2\n flag3=0\n init_v={init_v}        /\n")
    args = [DRIVER, "--bc", "0,0,0,0,0,0"] + (["--periodic-init"] if periodic else [])
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr + r.stdout
    a = orc.init_reference(init_v, l, m, n, periodic=periodic)
    p = orc.params(l, m, n, [0, 0, 0, 0, 0, 0], svisc=0.02)
    orc.run(p, a, None, 10)
    got, it = eup.read_raw_state(tmp_path / "save.00.00.00.00000010.bin", l, m, n)
    assert it == 10
    for q in range(19):
        assert np.array_equal(got[q], a[q]), q

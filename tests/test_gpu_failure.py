"""Failure detection through the C ABI, with every failure made on the host.

* A state holding a value that is not finite is refused at the boundary
  (eup_upload, eup_restore_state: EUP_ERR_INVALID_ARG) and leaves the handle
  without a state, so no step runs on it.
* A run that diverges is reported by the FP64 readers: eup_get_monitor,
  eup_get_forces, eup_get_force_series and eup_get_cd_series return
  EUP_ERR_DIVERGED once a sum or a force is not finite.  Two ways in: a finite
  but absurd state uploaded from the host (momentum 2e30 at one node two nodes
  upstream of the obstacle, which overflows the FP32 collision), and the cylinder channel at
  Re 2000 (tau = 0.5015), which the BGK collision cannot hold and which blows up
  by itself within a few thousand steps.

The reference has no such detection (CODE/SRC/diagno.F90:76-157 only sums);
hencol.F90:42-47 is its one sanity check, on the relaxation time.
No kernel is made to fault: NaN and Inf are ordinary floating-point values to
the step, whose memory accesses depend on node positions only.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIVERGED, INVALID = 4, 1


def _small_case(eup, precision=None):
    l, m, n = 48, 24, 8
    bc = (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    obs = eup.geometry_cylinder_z(l, m, n, 16, 12.5, 4)
    cfg = eup.Config(l, m, n, bc=bc, svisc=0.01, u_inflow=0.05, cd_uref=0.05, cd_length=8, cd_span=n,
                     precision=eup.FP32 if precision is None else precision)
    return cfg, obs


@pytest.mark.parametrize("where", ["interior", "halo"])
@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_upload_refuses_non_finite(eup, require_gpu, where, bad):
    cfg, obs = _small_case(eup)
    a = eup.init_equilibrium(cfg.lx, cfg.ly, cfg.lz, 0.05, 1e-4, 7, np.float32)
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(a)
        s.step(3)
        b = a.copy()
        if where == "interior":
            b[6, 4, 5, 20] = bad  # a07 at (20, 5, 4)
        else:
            b[13, 0, 3, 7] = bad  # a14 on the z = 0 halo plane
        with pytest.raises(eup.EupError) as ei:
            s.upload(b)
        assert ei.value.code == INVALID
        assert ("a7" if where == "interior" else "a14") in str(ei.value)
        # the rejected state is not stepped
        with pytest.raises(eup.EupError) as ei:
            s.step(1)
        assert ei.value.code == INVALID and "no state" in str(ei.value)
        # a good state is accepted again
        s.upload(a)
        s.step(1)
        assert np.isfinite(s.forces()).all()


def test_restore_refuses_non_finite(eup, require_gpu, tmp_path):
    cfg, obs = _small_case(eup)
    a = eup.init_equilibrium(cfg.lx, cfg.ly, cfg.lz, 0.05, 1e-4, 8, np.float32)
    a[2, 3, 3, 3] = np.nan
    path = str(tmp_path / "restore.bin")
    eup.write_raw_state(path, a, 10)
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        with pytest.raises(eup.EupError) as ei:
            s.restore_state(path, 4)
        assert ei.value.code == INVALID and "a3" in str(ei.value)


def _assert_diverged(eup, s, steps_done):
    with pytest.raises(eup.EupError) as ei:
        s.monitor()
    assert ei.value.code == DIVERGED
    with pytest.raises(eup.EupError) as ei:
        s.forces()
    assert ei.value.code == DIVERGED
    with pytest.raises(eup.EupError) as ei:
        s.cd_series(0, steps_done + 1)
    assert ei.value.code == DIVERGED
    with pytest.raises(eup.EupError) as ei:
        s.force_series(steps_done, 1)
    assert ei.value.code == DIVERGED


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_absurd_state_is_reported_diverged(eup, require_gpu, prec):
    cfg, obs = _small_case(eup, eup.FP32 if prec == "fp32" else eup.FP16_DEV)
    a = eup.init_equilibrium(cfg.lx, cfg.ly, cfg.lz, 0.05, 1e-4, 9, np.float32)
    # fluid node (i, j, k) = (11, 12, 4), two nodes upstream of the cylinder (centre (16, 12.5),
    # radius 4) and on no wall link: momentum 2e30 along x with the density unchanged, finite
    # in FP32 (infinite once stored as a 16-bit deviation), overflows in the collision
    assert obs[3, 11, 10] == 0 and obs[3, 11, 11] == 0 and obs[3, 11, 12] == 1
    a[0, 4, 12, 11] += 1e30   # a01, c = (1, -1, 0)
    a[11, 4, 12, 11] -= 1e30  # a12, its opposite
    assert np.isfinite(a).all()
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(a)  # finite: accepted
        f0 = s.forces()
        assert np.isfinite(f0).all()
        s.step(5)
        _assert_diverged(eup, s, 5)
        # the earlier, finite part of the history still reads back
        assert np.isfinite(s.force_series(0, 1)).all()


@pytest.mark.slow
def test_re2000_cylinder_channel_diverges_and_is_reported(eup, require_gpu):
    from euplectella_hpc_b200 import workloads
    wl = workloads.cylinder_channel(re=2000.0)
    assert abs(wl.cfg.svisc - 0.0005) < 1e-15
    with eup.Solver(wl.cfg) as s:
        s.set_obstacles(wl.obs)
        s.upload(wl.initial_state(np.float32))
        done, first_bad = 0, None
        while done < 6000:
            s.step(250)
            done += 250
            try:
                s.monitor()
            except eup.EupError as e:
                assert e.code == DIVERGED
                first_bad = done
                break
        assert first_bad is not None, "the Re 2000 run stayed finite for 6000 steps"
        s.step(400)  # let the non-finite values reach the cylinder's wall links
        _assert_diverged(eup, s, first_bad + 400)

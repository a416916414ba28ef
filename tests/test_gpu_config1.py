"""The cylinder channel of the plain reference method at its stated size and length,
run on the GPU through the C ABI against the CPU oracle.

Workload: 256x128x64 lattice nodes, a solid circular cylinder of diameter 20 with its
axis along z centred at (64, 64), uniform inlet u_x = 0.05 at x = 0 (rear, flag 4),
zero-gradient equilibrium outlet (front, flag 5), free-slip y, periodic z, halfway
bounce-back on the cylinder, Re 100 on the diameter (svisc 0.01), initial state the
equilibrium at rho = 1, u = inlet plus a seeded uniform perturbation of +-1e-4, 2000
steps.  The step being matched is CODE/SRC/bgk3d.F90:114-152 (bounce-back
bcond.obs.F90:47-77, halo planes bcond.bc.F90, streaming movef.F90:43-68, collision
col.F90:96-235).

* FP32 (the reference's native precision) and FP64: every fluid and halo value of the
  state after 2000 steps bit for bit against the float / double oracle; the obstacle mask, the link
  classification and the boundary-solid list exactly; the FP64 drag of each of the
  last 500 steps within 1e-12 and its time average within 0.1 %.
* FP16 and BF16 deviation storage against the FP64 run of the same kernel (held bit-exact
  with the double oracle on this very case above): velocity relative L2 over the
  fluid at step 2000 within 1e-3, C_d averaged over the last 500 steps within 0.5 %.
  BF16 misses the velocity bound (expected failure, with the measured value).
"""
import numpy as np
import pytest

from conftest import fluid_mask_haloed

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

STEPS = 2000
AVG = 500  # last quarter


@pytest.fixture(scope="module")
def wl(eup):
    from euplectella_hpc_b200 import workloads
    return workloads.cylinder_channel()


def _oracle_params(orc, wl):
    c = wl.cfg
    return orc.params(c.lx, c.ly, c.lz, c.bc, svisc=c.svisc, u0=c.u0, u_inflow=c.u_inflow, u00=c.u00)


def _cd_norm(wl):
    c = wl.cfg
    return 0.5 * c.cd_rho0 * c.cd_uref * c.cd_uref * c.cd_length * c.cd_span


def test_config1_geometry(eup, orc, require_gpu, wl):
    c = wl.cfg
    assert (c.lx, c.ly, c.lz) == (256, 128, 64)
    assert tuple(c.bc) == (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    assert abs(c.svisc - 0.05 * 20 / 100) < 1e-15
    # the disc (i - 64)^2 + (j - 64)^2 <= 10^2 on every z-plane, restated here
    k, j, i = np.meshgrid(np.arange(1, c.lz + 1), np.arange(1, c.ly + 1), np.arange(1, c.lx + 1), indexing="ij")
    disc = (((i - 64.0) ** 2 + (j - 64.0) ** 2) <= 100.0).astype(np.int32)
    assert np.array_equal(wl.obs, disc)
    p = _oracle_params(orc, wl)
    with eup.Solver(c) as s:
        s.build_obstacles(wl.geometry)  # voxelised on the device
        dev_obs, nobs = s.obstacles()
        assert np.array_equal(dev_obs, disc) and nobs == int(disc.sum())
        assert np.array_equal(s.links(), orc.links(p, disc))
        assert np.array_equal(s.boundary_solid(), orc.boundary_solid(p, disc))


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_config1_bit_exact_2000_steps(eup, orc, require_gpu, wl, prec):
    import dataclasses as dc
    dt, code = (np.float32, eup.FP32) if prec == "fp32" else (np.float64, eup.FP64)
    c = dc.replace(wl.cfg, precision=code)
    a0 = wl.initial_state(dt)
    with eup.Solver(c) as s:
        s.set_obstacles(wl.obs)
        s.upload(a0)
        s.step(STEPS)
        got = s.download(dt)
        f_gpu = s.force_series(STEPS - AVG + 1, AVG)
        cd_gpu = s.cd_series(STEPS - AVG + 1, AVG)
    p = _oracle_params(orc, wl)
    ref = a0.copy()
    b = np.empty_like(ref)
    orc.run(p, ref, wl.obs, STEPS - AVG, b)
    f_ref = np.empty((AVG, 3))
    for t in range(AVG):
        orc.run(p, ref, wl.obs, 1, b)
        f_ref[t] = orc.mem_force(p, ref, wl.obs)
    keep = fluid_mask_haloed(wl.obs)
    for q in range(19):
        bad = (got[q] != ref[q]) & keep
        assert not bad.any(), f"population {q + 1}: {bad.sum()} values differ, first at {np.argwhere(bad)[0]}"
    # FP64 sums over the wall links in another order
    np.testing.assert_allclose(f_gpu, f_ref, rtol=1e-12, atol=1e-12 * np.abs(f_ref).max())
    cd_ref = f_ref[:, 0] / _cd_norm(wl)
    np.testing.assert_allclose(cd_gpu, cd_ref, rtol=1e-12, atol=1e-12 * np.abs(cd_ref).max())
    assert abs(cd_gpu.mean() - cd_ref.mean()) <= 1e-3 * abs(cd_ref.mean())


def _run(eup, wl, precision, dtype):
    import dataclasses as dc
    cfg = dc.replace(wl.cfg, precision=precision)
    with eup.Solver(cfg) as s:
        s.set_obstacles(wl.obs)
        s.upload(wl.initial_state(np.float64))
        mass0 = s.monitor()[0]
        s.step(STEPS)
        state = s.download(np.float64)  # 16-bit storage expands to double exactly
        cd = s.cd_series(STEPS - AVG + 1, AVG)
        mass1 = s.monitor()[0]
    return state, cd, (mass1 - mass0) / mass0


@pytest.fixture(scope="module")
def fp64_run(eup, wl):
    if eup.device_count() == 0:
        pytest.fail("no CUDA device visible: -m gpu tests need a B200")
    return _run(eup, wl, eup.FP64, np.float64)


_runs16 = {}


def _errors(eup, wl, fp64_run, prec):
    if prec not in _runs16:
        code = eup.FP16_DEV if prec == "fp16" else eup.BF16_DEV
        s64, cd64, drift64 = fp64_run
        s16, cd16, drift16 = _run(eup, wl, code, np.float64)
        from euplectella_hpc_b200.studies import velocity
        fluid = wl.obs == 0
        u64, u16 = velocity(s64)[:, fluid], velocity(s16)[:, fluid]
        l2 = np.linalg.norm(u16 - u64) / np.linalg.norm(u64)
        cd_err = abs(cd16.mean() - cd64.mean()) / abs(cd64.mean())
        msg = (f"{prec}: velocity rel L2 {l2:.3e} (target 1e-3), C_d mean {cd16.mean():.6f} vs FP64 "
               f"{cd64.mean():.6f} = {cd_err:.3e} (target 5e-3), mass drift {drift16:.2e} (FP64 {drift64:.2e})")
        print(msg)
        _runs16[prec] = (l2, cd_err, msg)
    return _runs16[prec]


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_config1_16bit_cd_against_fp64(eup, require_gpu, wl, fp64_run, prec):
    _, cd_err, msg = _errors(eup, wl, fp64_run, prec)
    assert cd_err <= 5e-3, msg


# BF16 keeps 8 significand bits: a stored deviation is rounded to 2^-9 of itself, and on a
# B200 the velocity field after 2000 steps sits at relative L2 6.8e-3 from the FP64 run (C_d
# within 0.29 %, which passes above); FP16 (11 bits) sits at 3.4e-4.
@pytest.mark.parametrize("prec", [
    "fp16",
    pytest.param("bf16", marks=pytest.mark.xfail(strict=True, reason="BF16 storage misses the 1e-3 velocity L2 "
                                                 "target: 6.8e-3 measured at 2000 steps")),
])
def test_config1_16bit_velocity_against_fp64(eup, require_gpu, wl, fp64_run, prec):
    l2, _, msg = _errors(eup, wl, fp64_run, prec)
    assert l2 <= 1e-3, msg

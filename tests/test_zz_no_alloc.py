"""eup_mem_force_noalloc: the momentum-exchange force for callers that cannot
allocate device memory (a Fortran/OpenACC driver handing over its own
device-resident arrays, or a code with a fixed device-memory budget managed by its
own allocator).  It reads the
caller's device arrays, writes to the caller's device output, and uses only
the library's fixed scratch array.  Checked through the C ABI against
eup_get_forces on the same state, on two calls in a row.  This file is
collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(eup, l, m, n, bc, ptrs, elem_bytes, obs_ptr, out_ptr, stream):
    bcs = (ctypes.c_int32 * 6)(*bc)
    return eup.lib.eup_mem_force_noalloc(l, m, n, bcs, (ctypes.c_void_p * 19)(*ptrs), elem_bytes, obs_ptr,
                                         out_ptr, stream)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_noalloc_force_matches_handle(eup, require_gpu, prec):
    import torch

    l, m, n = 96, 40, 12
    bc = (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    dt, tdt, eb, code = ((np.float32, torch.float32, 4, eup.FP32) if prec == "fp32"
                         else (np.float64, torch.float64, 8, eup.FP64))
    obs = eup.geometry_cylinder_z(l, m, n, 30, 20.5, 6)
    cfg = eup.Config(l, m, n, bc=bc, svisc=0.01, u_inflow=0.05, precision=code)
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(eup.init_equilibrium(l, m, n, 0.05, 1e-3, 11, dt))
        s.step(30)
        f_ref = s.forces()
        state = s.download(dt)
    # caller-owned device memory (allocated here, by the caller, not by the entry point)
    dev = torch.device("cuda", 0)
    pops = torch.from_numpy(state).to(dev)
    d_obs = torch.from_numpy(obs).to(dev)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ptrs = [pops[q].data_ptr() for q in range(19)]
    for _ in range(2):
        out.fill_(float("nan"))
        rc = _call(eup, l, m, n, bc, ptrs, eb, d_obs.data_ptr(), out.data_ptr(), stream.cuda_stream)
        assert rc == 0, eup.lib.eup_last_error(None)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), f_ref, rtol=1e-12, atol=1e-14)
    del pops


def test_noalloc_on_a_caller_stream(eup, require_gpu):
    """The counter reset and the kernel run in order on a non-default stream of the caller."""
    import torch

    l, m, n = 64, 24, 10
    bc = (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    obs = eup.geometry_cylinder_z(l, m, n, 20, 12.5, 5)
    cfg = eup.Config(l, m, n, bc=bc, svisc=0.01, u_inflow=0.05)
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(eup.init_equilibrium(l, m, n, 0.05, 1e-3, 12, np.float32))
        s.step(20)
        f_ref = s.forces()
        state = s.download(np.float32)
    dev = torch.device("cuda", 0)
    side = torch.cuda.Stream(dev)
    with torch.cuda.stream(side):
        pops = torch.from_numpy(state).to(dev)
        d_obs = torch.from_numpy(obs).to(dev)
        out = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
        ptrs = [pops[q].data_ptr() for q in range(19)]
        for _ in range(2):
            out.fill_(float("nan"))
            rc = _call(eup, l, m, n, bc, ptrs, 4, d_obs.data_ptr(), out.data_ptr(), side.cuda_stream)
            assert rc == 0, eup.lib.eup_last_error(None)
            got = out.cpu().numpy()  # ordered after the kernel on the same stream
            np.testing.assert_allclose(got, f_ref, rtol=1e-12, atol=1e-14)
    side.synchronize()


def test_noalloc_rejects_oversized_lattice(eup):
    dummy = [1] * 19
    rc = _call(eup, 8, 8, 4097, (0,) * 6, dummy, 4, 1, 1, None)
    assert rc == 5
    assert b"4096" in eup.lib.eup_last_error(None)

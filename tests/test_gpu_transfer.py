"""State transfers through page-locked host memory.  eup_upload and eup_download move the 19
populations through two staging buffers, the host copy of one population on a copy stream
beside the scatter (gather) kernel of the one before, with events ordering each buffer's
reuse.  Copies from pageable arrays are synchronous, so only page-locked arrays exercise that
overlap: here transfers back to back, exact round trips in FP32/FP64, and the stepped state
equal, bit for bit, to the same run uploaded from a pageable array."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, M, N = 128, 64, 48


def _pinned(shape, dtype):
    import torch
    t = torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.float32, pin_memory=True)
    return t, t.numpy()


def _ptrs(a):
    return [a[q].ctypes.data for q in range(19)]


@pytest.mark.parametrize("prec", ["fp32", "fp64", "fp16"])
def test_page_locked_transfers_equal_pageable(eup, require_gpu, prec):
    code, dt = {"fp32": (eup.FP32, np.float32), "fp64": (eup.FP64, np.float64), "fp16": (eup.FP16_DEV, np.float32)}[prec]
    eb = np.dtype(dt).itemsize
    cfg = eup.Config(L, M, N, bc=(eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC),
                     svisc=0.01, u_inflow=0.05, precision=code)
    obs = eup.geometry_cylinder_z(L, M, N, 40, 32.5, 8)
    a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 21, dt)
    b = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 22, dt)
    keep = [_pinned(a.shape, dt) for _ in range(4)]  # tensors stay alive with their arrays
    src_a, src_b, out1, out2 = (k[1] for k in keep)
    src_a[...] = a
    src_b[...] = b
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload_ptrs(_ptrs(src_b), eb)  # a first state, overwritten at once: buffers reused back to back
        s.upload_ptrs(_ptrs(src_a), eb)
        s.download_ptrs(_ptrs(out1), eb)
        s.download_ptrs(_ptrs(out2), eb)
        if prec != "fp16":  # 16-bit storage rounds the deviations
            assert np.array_equal(out1, a)
        assert np.array_equal(out1, out2)
        s.step(6)
        s.download_ptrs(_ptrs(out1), eb)
        f = s.forces()
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(a)
        s.step(6)
        ref = s.download(dt)
        f_ref = s.forces()
    assert np.array_equal(out1, ref)
    assert np.array_equal(f, f_ref)

"""The staged 16-bit stream-collide kernel (pulls brought into shared memory by bulk
asynchronous copies, a ring of stages per persistent CTA; EUP_STEP_VARIANT=128, and 2176
for two CTAs per SM instead of three) against the register-pull two-node kernel (the
default), bit for bit, over lattice shapes that exercise its tiling: 512-node tiles that
cross rows, partial last tiles of a plane, one interior row or plane, no interior rows at
all (every row on a y/z boundary plane), rows shorter and longer than a tile."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(8, 5, 4), (16, 3, 3), (24, 11, 6), (256, 20, 13), (1024, 6, 5), (768, 7, 5), (40, 2, 5), (16, 9, 1),
          (512, 10, 4), (64, 33, 7)]


def _obs(l, m, n):
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    r = max(1.0, min(l, m) / 5)
    obs = ((i - l / 3) ** 2 + (j - (m + 1) / 2) ** 2 <= r * r).astype(np.int32)
    obs[:, :, l - 1] = 0  # none on the outflow plane
    return obs


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
@pytest.mark.parametrize("shape", SHAPES, ids=[f"{a}x{b}x{c}" for a, b, c in SHAPES])
@pytest.mark.parametrize("bc", [(5, 4, 3, 3, 0, 0), (0, 0, 0, 0, 0, 0)], ids=["channel", "periodic"])
def test_staged_equals_register_pull(eup, require_gpu, monkeypatch, prec, shape, bc):
    l, m, n = shape
    code = eup.FP16_DEV if prec == "fp16" else eup.BF16_DEV
    obs = _obs(l, m, n) if bc[0] == 5 else np.zeros((n, m, l), np.int32)
    a = eup.init_equilibrium(l, m, n, 0.05, 1e-3, 5, np.float64)
    cfg = eup.Config(l, m, n, bc=bc, svisc=0.01, u_inflow=0.05 if bc[0] == 5 else 0.0, precision=code)
    res = []
    for var in ("128", "0", "2176"):
        monkeypatch.setenv("EUP_STEP_VARIANT", var)
        with eup.Solver(cfg) as s:
            s.set_obstacles(obs)
            s.upload(a)
            s.step(9)
            s.synchronize()
            res.append((s.download(np.float64), s.force_series(0, 10)))
    for got, f in res[1:]:
        assert np.array_equal(res[0][0], got)
        assert np.array_equal(res[0][1], f)

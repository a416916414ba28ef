"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py):
the oracle must reproduce them bit for bit on the CPU, and the GPU path
through the C ABI must hit the same digests."""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
G = importlib.util.module_from_spec(spec)
spec.loader.exec_module(G)

NAMES = sorted(G.FIXTURES)


def load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(orc, name):
    ref = load(name)
    got = G.generate(name)
    assert np.array_equal(got["obs"], ref["obs"])
    for key in ("sha_init", "sha_step1", "sha_step10", "sha_step40"):
        assert str(got[key]) == str(ref[key]), key
    assert np.array_equal(got["forces"], ref["forces"])
    if "state_step10" in ref:
        assert np.array_equal(got["state_step10"], ref["state_step10"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_fixture(eup, require_gpu, name):
    ref = load(name)
    l, m, n, bc, svisc, uin, _spec, dt = G.FIXTURES[name]
    obs = ref["obs"]
    a = eup.init_equilibrium(l, m, n, uin, 1e-3, G.SEED, dt)
    assert G.digest(a, obs) == str(ref["sha_init"])
    prec = eup.FP64 if dt == np.float64 else eup.FP32
    with eup.Solver(eup.Config(l, m, n, bc=bc, svisc=svisc, u_inflow=uin, precision=prec)) as s:
        s.set_obstacles(obs)
        s.upload(a)
        done = 0
        for t in G.SNAPSHOTS:
            s.step(t - done)
            done = t
            got = s.download(dt)
            if t == 10 and "state_step10" in ref:
                diff = G.masked(got, obs) != ref["state_step10"]
                assert not diff.any(), f"{diff.sum()} values differ at step 10"
            assert G.digest(got, obs) == str(ref[f"sha_step{t}"]), t
        f = s.force_series(0, max(G.SNAPSHOTS) + 1)
    np.testing.assert_allclose(f, ref["forces"], rtol=1e-12, atol=1e-14)

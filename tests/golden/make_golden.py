"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference ships no golden vectors, so these fixtures pin the oracle (the
C restatement of the reference's serial step) against itself over time, and
give the GPU tests a stored target.  Each fixture holds SHA-256 digests of the
seeded initial state and of the haloed state after 1, 10 and 40 steps (interior
solid voxels zeroed: their values are not part of the reference's observable
result), the FP64 momentum-exchange force of every step, and the full masked
state after 10 steps for diagnosing a mismatch.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# name: (l, m, n, bc, svisc, u_inflow, obstacle spec, dtype)
FIXTURES = {
    "cyl_freeslipY_periodicZ_f32": (16, 12, 6, (5, 4, 3, 3, 0, 0), 0.01, 0.05, ("cyl", 5.5, 6.5, 2.2), np.float32),
    "shell_freeslip_all_f32": (16, 10, 10, (5, 4, 3, 3, 3, 3), 0.0024, 0.05, ("box", 5, 8, 3, 7, 3, 7), np.float32),
    "cyl_freeslipY_periodicZ_f64": (16, 12, 6, (5, 4, 3, 3, 0, 0), 0.01, 0.05, ("cyl", 5.5, 6.5, 2.2), np.float64),
}
SNAPSHOTS = (1, 10, 40)
SEED = 1234


def obstacle(spec, l, m, n):
    obs = np.zeros((n, m, l), np.int32)
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    if spec[0] == "cyl":
        _, xc, yc, r = spec
        obs[((i - xc) ** 2 + (j - yc) ** 2) <= r * r] = 1
    else:
        _, i0, i1, j0, j1, k0, k1 = spec
        obs[(i >= i0) & (i <= i1) & (j >= j0) & (j <= j1) & (k >= k0) & (k <= k1)] = 1
        obs[(i > i0) & (i < i1) & (j > j0) & (j < j1) & (k > k0) & (k < k1)] = 0  # hollow box
    return obs


def masked(a, obs):
    """Copy of the haloed state with interior solid voxels set to zero."""
    out = a.copy()
    out[:, 1:-1, 1:-1, 1:-1][:, obs == 1] = 0
    return out


def digest(a, obs):
    return hashlib.sha256(np.ascontiguousarray(masked(a, obs)).tobytes()).hexdigest()


def generate(name):
    l, m, n, bc, svisc, uin, spec, dt = FIXTURES[name]
    obs = obstacle(spec, l, m, n)
    p = O.params(l, m, n, bc, svisc=svisc, u_inflow=uin)
    a = O.init_perturbed(l, m, n, uin, 1e-3, SEED, dt)
    out = {"sha_init": np.array(digest(a, obs)), "obs": obs}
    forces = [O.mem_force(p, a, obs)]
    b = np.zeros_like(a)
    for t in range(1, max(SNAPSHOTS) + 1):
        O.run(p, a, obs, 1, b)
        forces.append(O.mem_force(p, a, obs))
        if t in SNAPSHOTS:
            out[f"sha_step{t}"] = np.array(digest(a, obs))
        if t == 10 and dt == np.float32:
            out["state_step10"] = masked(a, obs)
    out["forces"] = np.array(forces)
    return out


def main():
    for name in FIXTURES:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **generate(name))
        print("wrote", name)


if __name__ == "__main__":
    main()

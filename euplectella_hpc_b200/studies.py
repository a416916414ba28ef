"""Precision study: populations stored as scaled deviations (f_q - w_q) in FP16
and in BF16 with FP32 arithmetic (and plain FP32), each measured against an
FP64 run of the same kernel on the same geometry, inputs and step count.

Default: the 256x128x64 channel with a D=20 cylinder (inflow 0.05, outflow,
free-slip y, periodic z) at Re in {500, 1000, 2000}, 20000 steps each.  For
every run: velocity relative L2 over fluid nodes at the last step, relative
error of the time-averaged C_d over the last quarter of the run, relative
difference of the FP64 mass sum at the last step, and the device time.

    python -m euplectella_hpc_b200.studies [--steps N] [--re 500,1000,2000] [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import BF16_DEV, FP16_DEV, FP32, FP64, EupError, Solver
from .workloads import cylinder_channel

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], dtype=np.float64)
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], dtype=np.float64)
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], dtype=np.float64)


def velocity(pops: np.ndarray) -> np.ndarray:
    c = pops[:, 1:-1, 1:-1, 1:-1].astype(np.float64)
    rho = c.sum(0)
    return np.stack([np.tensordot(CX, c, 1), np.tensordot(CY, c, 1), np.tensordot(CZ, c, 1)]) / rho


def run_one(wl, precision, steps, chunk=1000):
    """Runs `steps` steps; returns final state (float64), C_d series, mass, device seconds, diverged step."""
    wl.cfg.precision = precision
    a = wl.initial_state(np.float64)
    cd = np.zeros(steps + 1)
    diverged = None
    with Solver(wl.cfg) as s:
        s.set_obstacles(wl.obs)
        s.upload(a)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(chunk, steps - done)
            s.step(k)
            s.synchronize()
            cd[done + 1:done + k + 1] = s.cd_series(done + 1, k)
            done += k
            try:
                s.monitor()
            except EupError:
                diverged = done
                break
        dt = time.perf_counter() - t0
        mass = s.monitor()[0] if diverged is None else float("nan")
        state = s.download(np.float64)
    return state, cd[:done + 1], mass, dt, diverged


def precision_study(re_list=(500.0, 1000.0, 2000.0), steps=20000):
    rows = []
    for re in re_list:
        wl = cylinder_channel(re=re, steps=steps)
        fluid = wl.obs == 0
        ref_state, ref_cd, ref_mass, ref_dt, ref_div = run_one(wl, FP64, steps)
        v_ref = velocity(ref_state)[:, fluid]
        tail = slice(3 * steps // 4, steps + 1)
        for name, prec in (("fp32", FP32), ("fp16-dev", FP16_DEV), ("bf16-dev", BF16_DEV)):
            st, cd, mass, dt, div = run_one(wl, prec, steps)
            row = {"re": re, "storage": name, "steps": steps, "nu": wl.cfg.svisc,
                   "fp64_diverged_at": ref_div, "diverged_at": div, "seconds": dt, "fp64_seconds": ref_dt}
            if div is None and ref_div is None:
                v = velocity(st)[:, fluid]
                row["velocity_rel_l2"] = float(np.linalg.norm(v - v_ref) / np.linalg.norm(v_ref))
                row["cd_mean"] = float(cd[tail].mean())
                row["cd_mean_fp64"] = float(ref_cd[tail].mean())
                row["cd_rel_err"] = abs(row["cd_mean"] - row["cd_mean_fp64"]) / abs(row["cd_mean_fp64"])
                row["mass_rel_diff"] = float(abs(mass - ref_mass) / ref_mass)
            rows.append(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--re", default="500,1000,2000")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    rows = precision_study(tuple(float(x) for x in args.re.split(",")), args.steps)
    for r in rows:
        print(json.dumps(r))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()

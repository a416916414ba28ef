"""Precision study: populations stored as scaled deviations (f_q - w_q) in FP16
and in BF16 with FP32 arithmetic (and plain FP32), each measured against an
FP64 run of the same kernel on the same geometry, inputs and step count.

Default: the 256x128x64 channel with a D=20 cylinder (inflow 0.05, outflow,
free-slip y, periodic z) at Re in {500, 1000, 2000}, 20000 steps each.  For
every run: velocity relative L2 over fluid nodes at the last step, relative
error of the time-averaged C_d over the last quarter of the run, relative
difference of the FP64 mass sum at the last step, and the device time.

    python -m euplectella_hpc_b200.studies [--steps N] [--re 500,1000,2000] [--out FILE]

Adjoint study (config 4): python -m euplectella_hpc_b200.studies --adjoint --steps 4000 [--fd 32]
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


def adjoint_study(steps=4000, avg_steps=1000, checkpoints=64, n_fd=32, h=1e-3, fd_seed=2027):
    """Config-4 adjoint: mean C_d over the last avg_steps of `steps` on the 192x96x96 partial-
    bounce-back channel.  Returns timings (adjoint with recomputation vs a plain forward run of the
    same steps), the FP32-vs-FP64 adjoint gradient difference, and central finite differences of
    FP64 forward runs at n_fd seeded voxels against the FP64 adjoint."""
    from .workloads import pbb_cylinder_channel
    out = {"steps": steps, "avg_steps": avg_steps, "checkpoints": checkpoints}
    grads = {}
    for name, prec, dt in (("fp32", FP32, np.float32), ("fp64", FP64, np.float64)):
        wl = pbb_cylinder_channel(steps=steps, avg_steps=avg_steps, precision=prec)
        a = wl.initial_state(dt)
        with Solver(wl.cfg) as s:
            s.set_solid_fraction(wl.ns)
            s.upload(a)
            fwd_ms = s.step_profiled(steps)[3]
        with Solver(wl.cfg) as s:
            s.set_solid_fraction(wl.ns)
            s.upload(a)
            J, g, st = s.adjoint(steps, avg_steps, checkpoints)
        grads[name] = g
        out[name] = {"objective": J, "forward_ms": fwd_ms, "adjoint_forward_sweep_ms": st["forward_ms"],
                     "adjoint_reverse_ms": st["reverse_ms"],
                     "adjoint_over_forward": (st["forward_ms"] + st["reverse_ms"]) / fwd_ms,
                     "recomputed_steps": st["recomputed_steps"], "checkpoints_used": st["checkpoints"],
                     "segment_steps": st["segment_steps"], "stored_state_bytes": st["state_bytes"]}
    out["grad_fp32_vs_fp64_rel_l2"] = float(np.linalg.norm(grads["fp32"] - grads["fp64"]) /
                                            np.linalg.norm(grads["fp64"]))
    # central differences (FP64) at seeded voxels away from the [0,1] bounds
    wl = pbb_cylinder_channel(steps=steps, avg_steps=avg_steps, precision=FP64)
    a = wl.initial_state(np.float64)
    norm = 0.5 * wl.cfg.cd_rho0 * wl.cfg.cd_uref ** 2 * wl.cfg.cd_length * wl.cfg.cd_span

    def objective(ns):
        with Solver(wl.cfg) as s:
            s.set_solid_fraction(ns)
            s.upload(a)
            s.step(steps)
            return s.force_series(steps - avg_steps + 1, avg_steps)[:, 0].mean() / norm

    rng = np.random.default_rng(fd_seed)
    cand = np.argwhere((wl.ns > h) & (wl.ns < 1 - h))
    pick = cand[rng.choice(len(cand), n_fd, replace=False)]
    rows = []
    for k, j, i in pick:
        p, m = wl.ns.copy(), wl.ns.copy()
        p[k, j, i] += h
        m[k, j, i] -= h
        fd = (objective(p) - objective(m)) / (2 * h)
        ad = float(grads["fp64"][k, j, i])
        rows.append({"voxel": [int(i) + 1, int(j) + 1, int(k) + 1], "ns": float(wl.ns[k, j, i]), "fd": fd,
                     "adjoint": ad, "rel_err": abs(ad - fd) / max(abs(fd), 1e-300)})
    out["fd"] = rows
    errs = np.array([r["rel_err"] for r in rows])
    out["fd_rel_err_max"] = float(errs.max())
    out["fd_rel_err_median"] = float(np.median(errs))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--re", default="500,1000,2000")
    ap.add_argument("--out", default=None)
    ap.add_argument("--adjoint", action="store_true", help="run the config-4 adjoint study instead")
    ap.add_argument("--fd", type=int, default=32)
    args = ap.parse_args()
    if args.adjoint:
        res = adjoint_study(steps=args.steps, n_fd=args.fd)
        print(json.dumps(res))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)
        return
    rows = precision_study(tuple(float(x) for x in args.re.split(",")), args.steps)
    for r in rows:
        print(json.dumps(r))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()

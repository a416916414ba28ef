"""Precision study: populations stored as scaled deviations (f_q - w_q) in FP16
and in BF16 with FP32 arithmetic (and plain FP32), each measured against an
FP64 run of the same kernel on the same geometry, inputs and step count.

Default: the 256x128x64 channel with a D=20 cylinder (inflow 0.05, outflow,
free-slip y, periodic z) at Re in {500, 1000, 2000}, 20000 steps each.  For
every run: velocity relative L2 over fluid nodes at the last step, relative
error of the time-averaged C_d over the last quarter of the run, relative
difference of the FP64 mass sum at the last step, and the device time.

    python -m euplectella_hpc_b200.studies [--steps N] [--re 500,1000,2000] [--out FILE]

Adjoint study (192x96x96 partial bounce-back channel):
    python -m euplectella_hpc_b200.studies --adjoint --steps 4000 [--fd 32]
Production forward runs: python -m euplectella_hpc_b200.studies --production shell|ridged [--steps N]
Ridge-height gradient:    python -m euplectella_hpc_b200.studies --ridge-adjoint
Obstacle masks, host voxeliser + eup_set_obstacles against eup_build_obstacles:
                          python -m euplectella_hpc_b200.studies --voxelise
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import time

import numpy as np

from . import BF16_DEV, FP16_DEV, FP32, FP64, EupError, Solver, voxelise
from .workloads import cylinder_channel

CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0], dtype=np.float64)
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0], dtype=np.float64)
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0], dtype=np.float64)


def velocity(pops: np.ndarray) -> np.ndarray:
    c = pops[:, 1:-1, 1:-1, 1:-1].astype(np.float64)
    rho = c.sum(0)
    return np.stack([np.tensordot(CX, c, 1), np.tensordot(CY, c, 1), np.tensordot(CZ, c, 1)]) / rho


def run_one(wl, precision, steps, chunk=500, samples=10, window=None):
    """Runs `steps` steps; returns final state (float64), C_d series, mass, seconds, diverged step and
    the velocity field averaged over `samples` snapshots evenly spaced in the last `window` steps
    (default the last quarter)."""
    wl.cfg.precision = precision
    a = wl.initial_state(np.float64)
    cd = np.zeros(steps + 1)
    diverged = None
    first = steps - (window if window else steps // 4)
    marks = set(int(round(first + (steps - first) * (t + 1) / samples)) for t in range(samples))
    vsum, nsum = None, 0
    with Solver(wl.cfg) as s:
        s.set_obstacles(wl.obs)
        s.upload(a)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            nxt = min([m for m in marks if m > done] + [done + chunk, steps])
            k = nxt - done
            s.step(k)
            s.synchronize()
            cd[done + 1:done + k + 1] = s.cd_series(done + 1, k)
            done += k
            try:
                s.monitor()
            except EupError:
                diverged = done
                break
            if done in marks:
                v = velocity(s.download(np.float64))
                vsum = v if vsum is None else vsum + v
                nsum += 1
        dt = time.perf_counter() - t0
        mass = s.monitor()[0] if diverged is None else float("nan")
        state = s.download(np.float64)
    vmean = vsum / nsum if nsum else None
    return state, cd[:done + 1], mass, dt, diverged, vmean


def precision_study(re_list=(500.0, 1000.0, 2000.0), steps=20000):
    rows = []
    for re in re_list:
        wl = cylinder_channel(re=re, steps=steps)
        fluid = wl.obs == 0
        ref_state, ref_cd, ref_mass, ref_dt, ref_div, ref_vm = run_one(wl, FP64, steps)
        v_ref = velocity(ref_state)[:, fluid]
        tail = slice(3 * steps // 4, steps + 1)
        for name, prec in (("fp32", FP32), ("fp16-dev", FP16_DEV), ("bf16-dev", BF16_DEV)):
            st, cd, mass, dt, div, vm = run_one(wl, prec, steps)
            row = {"re": re, "storage": name, "steps": steps, "nu": wl.cfg.svisc,
                   "fp64_diverged_at": ref_div, "diverged_at": div, "seconds": dt, "fp64_seconds": ref_dt}
            if div is None and ref_div is None:
                v = velocity(st)[:, fluid]
                row["velocity_rel_l2"] = float(np.linalg.norm(v - v_ref) / np.linalg.norm(v_ref))
                # time-averaged field over the last quarter: the comparison that stays meaningful
                # once the flow is unsteady and individual snapshots decorrelate
                vm_f, vr_f = vm[:, fluid], ref_vm[:, fluid]
                row["mean_velocity_rel_l2"] = float(np.linalg.norm(vm_f - vr_f) / np.linalg.norm(vr_f))
                row["cd_mean"] = float(cd[tail].mean())
                row["cd_mean_fp64"] = float(ref_cd[tail].mean())
                row["cd_rel_err"] = abs(row["cd_mean"] - row["cd_mean_fp64"]) / abs(row["cd_mean_fp64"])
                row["mass_rel_diff"] = float(abs(mass - ref_mass) / ref_mass)
            rows.append(row)
    return rows


def chaos_study(re_list=(500.0, 1000.0), steps=20000, avg_steps=10000, seeds=(1234, 1235, 1236, 1237),
                samples=10):
    """Storage error against the chaos floor.  For each Re, every storage format (FP64, FP32,
    FP16 and BF16 deviations) runs the 256x128x64 cylinder channel from `seeds` (the same
    equilibrium start with different seeded +-1e-4 perturbations): C_d averaged over the last
    avg_steps steps and the velocity field averaged over `samples` snapshots of that window.
    The spread of the FP64 runs over the seeds is what the flow's own sensitivity does to these
    averages; a storage format whose ensemble mean sits within that spread of the FP64 mean has
    an error below the chaos floor at this averaging length."""
    rows = []
    for re in re_list:
        wl = cylinder_channel(re=re, steps=steps)
        fluid = wl.obs == 0
        ens = {}
        for name, prec in (("fp64", FP64), ("fp32", FP32), ("fp16-dev", FP16_DEV), ("bf16-dev", BF16_DEV)):
            cds, vms = [], []
            for seed in seeds:
                wl.seed = seed
                _, cd, _, _, div, vm = run_one(wl, prec, steps, samples=samples, window=avg_steps)
                if div is not None:
                    cds.append(float("nan"))
                    vms.append(None)
                    continue
                cds.append(float(cd[steps - avg_steps + 1:].mean()))
                vms.append(vm[:, fluid])
            ens[name] = (np.array(cds), vms)
        cd64, v64 = ens["fp64"]
        vbar64 = np.mean([v for v in v64 if v is not None], axis=0)
        spread = float(np.std(cd64, ddof=1) / abs(np.mean(cd64)))
        v_spread = float(np.mean([np.linalg.norm(v - vbar64) / np.linalg.norm(vbar64) for v in v64]))
        for name, (cds, vms) in ens.items():
            ok = [v for v in vms if v is not None]
            row = {"re": re, "storage": name, "steps": steps, "avg_steps": avg_steps, "seeds": list(seeds),
                   "cd_mean_per_seed": cds.tolist(), "cd_ensemble_mean": float(np.nanmean(cds)),
                   "cd_ensemble_rel_std": float(np.nanstd(cds, ddof=1) / abs(np.nanmean(cds))),
                   "fp64_cd_rel_std": spread, "fp64_mean_velocity_spread": v_spread,
                   "cd_rel_diff_vs_fp64_ensemble": float(abs(np.nanmean(cds) - np.mean(cd64)) / abs(np.mean(cd64))),
                   "cd_rel_diff_same_seed": float(np.nanmean(np.abs(cds - cd64) / np.abs(cd64)))}
            if ok:
                vbar = np.mean(ok, axis=0)
                row["mean_velocity_rel_l2_vs_fp64_ensemble"] = float(np.linalg.norm(vbar - vbar64) / np.linalg.norm(vbar64))
            rows.append(row)
    return rows


def adjoint_study(steps=4000, avg_steps=1000, checkpoints=64, n_fd=32, h=1e-3, h_small=1e-5, fd_seed=2027):
    """Adjoint of mean C_d over the last avg_steps of `steps` on the 192x96x96 partial-
    bounce-back channel.  Returns timings (adjoint with recomputation vs a plain forward run of the
    same steps), the FP32-vs-FP64 adjoint gradient difference, and central finite differences of
    FP64 forward runs (steps h and h_small) at n_fd seeded voxels against the FP64 adjoint."""
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
                     "repetitions": st["repetitions"], "stored_state_bytes": st["state_bytes"]}
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

    def central(k, j, i, step):
        p, m = wl.ns.copy(), wl.ns.copy()
        p[k, j, i] += step
        m[k, j, i] -= step
        return (objective(p) - objective(m)) / (2 * step)

    for k, j, i in pick:
        fd = central(k, j, i, h)
        # a second, smaller step: where n_s is close to 1 the response is nonlinear enough that
        # the step-h difference carries a visible truncation error
        fd_small = central(k, j, i, h_small)
        ad = float(grads["fp64"][k, j, i])
        rows.append({"voxel": [int(i) + 1, int(j) + 1, int(k) + 1], "ns": float(wl.ns[k, j, i]), "fd": fd,
                     "fd_small_step": fd_small, "adjoint": ad, "rel_err": abs(ad - fd) / max(abs(fd), 1e-300),
                     "rel_err_small_step": abs(ad - fd_small) / max(abs(fd_small), 1e-300)})
    out["fd"] = rows
    out["fd_step"], out["fd_small_step"] = h, h_small
    # error relative to the sample's gradient scale: a component orders of magnitude below the
    # others is resolved by the central difference only to its truncation error
    for key, suffix in (("fd", ""), ("fd_small_step", "_small_step")):
        scale = 1e-3 * max(abs(r[key]) for r in rows)
        for r in rows:
            r["rel_err_scaled" + suffix] = abs(r["adjoint"] - r[key]) / max(abs(r[key]), scale)
        errs = np.array([r["rel_err" + suffix] for r in rows])
        out["fd_rel_err_max" + suffix] = float(errs.max())
        out["fd_rel_err_median" + suffix] = float(np.median(errs))
        out["fd_rel_err_scaled_max" + suffix] = float(max(r["rel_err_scaled" + suffix] for r in rows))
        out["fd_voxels_within_1e-3" + suffix] = int(sum(r["rel_err_scaled" + suffix] <= 1e-3 for r in rows))
    return out


def hbm_peak_gbs():
    """HBM copy bandwidth measured on this machine's B200 (MEASURED_PEAKS.json), else an earlier
    B200 copy measurement (6650 GB/s)."""
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def production_run(which="shell", steps=None, precision=None, chunk=1000):
    """Forward run of a production case from the seeded device-side initial state: the
    768x384x384 reticular shell (FP32, 20000 steps) or the 1024x512x512 ridged shell (FP16
    deviations, 10000 steps).  Reports MLUPS (wall time of the stepping, synchronised every
    chunk), the stream-collide kernel's fraction of the HBM roofline (CUDA-event phase times of
    a profiled window), C_d averaged over the last quarter, the probe velocities and the mean
    velocity inside the body cavity at the end."""
    from .workloads import U_IN, PERTURBATION, reticular_shell_channel, ridged_shell_channel
    if which == "shell":
        wl = reticular_shell_channel(precision=FP32 if precision is None else precision, host_mask=False)
    else:
        wl = ridged_shell_channel(precision=FP16_DEV if precision is None else precision, host_mask=False)
    steps = wl.steps if steps is None else steps
    c = wl.cfg
    sbytes = {FP32: 4, FP64: 8, FP16_DEV: 2, BF16_DEV: 2}[c.precision]
    peak, peak_kind = hbm_peak_gbs()
    out = {"workload": wl.name, "nodes": wl.nodes, "steps": steps, "precision": c.precision, "nu": c.svisc}
    cd = np.zeros(steps + 1)
    with Solver(c) as s:
        s.build_obstacles(wl.geometry)  # voxelised on the device: no host mask, no mask copy
        out["solid_voxels"] = s.obstacle_count()
        s.init_state(U_IN, PERTURBATION, wl.seed)
        done, wall = 0, 0.0
        while done < steps:
            k = min(chunk, steps - done)
            t0 = time.perf_counter()
            s.step(k)
            s.synchronize()
            wall += time.perf_counter() - t0
            cd[done + 1:done + k + 1] = s.cd_series(done + 1, k)
            done += k
            try:
                s.monitor()
            except EupError:
                out["diverged_at"] = done
                break
        out["wall_s"] = wall
        out["mlups"] = wl.nodes * done / wall / 1e6
        if "diverged_at" not in out:
            ph = s.step_profiled(50)
            kern_ms = ph[2] / 50
            out["stream_collide_ms"] = kern_ms
            out["stream_collide_gbs"] = 2 * 19 * sbytes * wl.nodes / (kern_ms * 1e-3) / 1e9
            out["hbm_peak_gbs"] = peak
            out["hbm_peak_kind"] = peak_kind
            out["roofline_frac"] = out["stream_collide_gbs"] / peak
            tail = slice(3 * done // 4, done + 1)
            out["cd_mean_last_quarter"] = float(cd[tail].mean())
            out["cd_std_last_quarter"] = float(cd[tail].std())
            out["cd_series_every_100"] = [float(x) for x in cd[:done + 1:100]]
            out["probes_rho_u"] = s.probes(wl.probes).tolist()
            if wl.cavity is not None:
                cav = np.broadcast_to(wl.cavity, (c.lz, c.ly, c.lx))
                r = s.region_sums(cav)
                out["cavity_nodes"] = int(r[0])
                out["cavity_mean_u"] = [float(r[2] / r[0]), float(r[3] / r[0]), float(r[4] / r[0])]
            out["mass"] = float(s.monitor()[0])
    return out


def ridge_adjoint(scale=0.25, re=500.0, steps=2500, avg_steps=625, checkpoints=64, smooth_w=0.5, dh=0.01,
                  precision=FP64):
    """Gradient of mean C_d with respect to the ridge height of the ridged shell, chained through
    the solid-fraction field: dJ/dh = sum_x dJ/dn_s(x) dn_s(x)/dh, with n_s = 1 on the shell and
    the cap and the ridges' radial extent smoothed over smooth_w, checked against a central
    difference of J in h (two forward runs).  Defaults: the scaled geometry (scale 1/4:
    256x128x128, shell D 24, ridges 2 lu) at the lattice viscosity of the full-size case (Re 500
    on the scaled diameter).  The full-size case is scale 1, Re 2000, 16-bit storage,
    10000 steps (python -m euplectella_hpc_b200.studies --ridge-adjoint --scale 1 --re 2000
    --precision fp16 --steps 10000 --checkpoints 8)."""
    from .workloads import U_IN, PERTURBATION, ridged_shell_channel
    wl = ridged_shell_channel(scale=scale, re=re, precision=precision)
    c = wl.cfg
    body = wl.body
    ns, dns = body.field(c.lx, c.ly, c.lz, smooth_w)
    norm = 0.5 * c.cd_rho0 * c.cd_uref ** 2 * c.cd_length * c.cd_span
    out = {"workload": wl.name, "scale": scale, "re": re, "nu": c.svisc, "steps": steps, "avg_steps": avg_steps,
           "ridge_h": body.ridge_h, "smooth_w": smooth_w, "dh": dh, "precision": precision}
    with Solver(c) as s:
        s.set_solid_fraction(ns)
        s.init_state(U_IN, PERTURBATION, wl.seed)
        fwd_ms = s.step_profiled(steps)[3]
    with Solver(c) as s:
        s.set_solid_fraction(ns)
        s.init_state(U_IN, PERTURBATION, wl.seed)
        J, g, st = s.adjoint(steps, avg_steps, checkpoints)
    out.update({"objective": J, "forward_ms": fwd_ms, "adjoint_ms": st["forward_ms"] + st["reverse_ms"],
                "adjoint_over_forward": (st["forward_ms"] + st["reverse_ms"]) / fwd_ms,
                "checkpoints_used": st["checkpoints"], "repetitions": st["repetitions"],
                "recomputed_steps": st["recomputed_steps"], "stored_state_bytes": st["state_bytes"],
                "nodes": c.lx * c.ly * c.lz, "partial_voxels": int((ns > 0).sum()),
                "grad_abs_max": float(np.abs(g).max()), "grad_finite": bool(np.isfinite(g).all())})
    out["dJ_dh_adjoint"] = float((g * dns).sum())
    del g

    def objective(h):
        f, _ = body.field(c.lx, c.ly, c.lz, smooth_w, ridge_h=h)
        with Solver(c) as s2:
            s2.set_solid_fraction(f)
            s2.init_state(U_IN, PERTURBATION, wl.seed)
            s2.step(steps)
            return s2.force_series(steps - avg_steps + 1, avg_steps)[:, 0].mean() / norm

    jp, jm = objective(body.ridge_h + dh), objective(body.ridge_h - dh)
    out["dJ_dh_central_difference"] = (jp - jm) / (2 * dh)
    out["rel_err"] = abs(out["dJ_dh_adjoint"] - out["dJ_dh_central_difference"]) / abs(out["dJ_dh_central_difference"])
    return out


def voxelise_timing(repeats=3):
    """The production obstacle masks (768x384x384 reticular shell, 1024x512x512 ridged shell)
    built and installed two ways, best of `repeats` wall times: the host voxeliser (OpenMP, all
    host threads) followed by eup_set_obstacles, which copies the int32 mask (4 B per node) to
    the device and packs it; and eup_build_obstacles, which voxelises on the device into the
    packed mask.  Also the obstacle file: eup_write_obs_file from the host mask against
    eup_write_obstacles, listed on the device."""
    import tempfile
    from . import lib
    from .workloads import reticular_shell_channel, ridged_shell_channel
    rows = []
    for wl in (reticular_shell_channel(host_mask=False), ridged_shell_channel(host_mask=False)):
        c = dataclasses.replace(wl.cfg, precision=FP16_DEV)
        row = {"workload": wl.name, "nodes": wl.nodes, "host_threads": os.cpu_count()}
        t_dev, t_vox, t_set, t_wdev, t_whost = [], [], [], [], []
        with Solver(c) as s, tempfile.TemporaryDirectory() as tmp:
            s.build_obstacles(wl.geometry)  # warm-up: first allocations, module load
            for _ in range(repeats):
                t0 = time.perf_counter()
                s.build_obstacles(wl.geometry)
                t_dev.append(time.perf_counter() - t0)
            row["solid_voxels"] = s.obstacle_count()
            for _ in range(repeats):
                t0 = time.perf_counter()
                obs = voxelise(wl.geometry, c.lx, c.ly, c.lz)
                t1 = time.perf_counter()
                s.set_obstacles(obs)
                t_vox.append(t1 - t0)
                t_set.append(time.perf_counter() - t1)
            path = os.path.join(tmp, "obs.bin")
            for _ in range(repeats):
                t0 = time.perf_counter()
                s.write_obstacles(path)
                t_wdev.append(time.perf_counter() - t0)
                t0 = time.perf_counter()
                lib.eup_write_obs_file(path.encode(), c.lx, c.ly, c.lz, obs.ctypes.data)
                t_whost.append(time.perf_counter() - t0)
        row.update(device_build_s=min(t_dev), host_voxelise_s=min(t_vox), host_set_obstacles_s=min(t_set),
                   host_total_s=min(a + b for a, b in zip(t_vox, t_set)), device_write_s=min(t_wdev),
                   host_write_s=min(t_whost))
        rows.append(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--re", default="500,1000,2000")
    ap.add_argument("--out", default=None)
    ap.add_argument("--adjoint", action="store_true", help="run the 192x96x96 partial-bounce-back adjoint study instead")
    ap.add_argument("--chaos", action="store_true",
                    help="storage error against the chaos floor: seed ensembles per storage format (--re, --steps)")
    ap.add_argument("--fd", type=int, default=32)
    ap.add_argument("--production", choices=["shell", "ridged"], default=None,
                    help="forward run of the 768x384x384 reticular shell or the 1024x512x512 ridged shell")
    ap.add_argument("--ridge-adjoint", action="store_true", help="ridge-height gradient on the scaled ridged shell")
    ap.add_argument("--precision", choices=["fp32", "fp64", "fp16", "bf16"], default=None,
                    help="storage of a production run (default: the case's own)")
    ap.add_argument("--chunk", type=int, default=1000, help="steps between divergence checks of a production run")
    ap.add_argument("--voxelise", action="store_true", help="time the production obstacle masks, host against device")
    ap.add_argument("--scale", type=float, default=0.25, help="ridge adjoint: geometry scale (1 = 1024x512x512)")
    ap.add_argument("--checkpoints", type=int, default=64, help="ridge adjoint: stored states")
    ap.add_argument("--avg", type=int, default=None, help="ridge adjoint: averaging window (default steps/4)")
    ap.add_argument("--dh", type=float, default=0.01, help="ridge adjoint: central-difference step in h")
    args = ap.parse_args()
    if args.voxelise:
        rows = voxelise_timing()
        for r in rows:
            print(json.dumps(r))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(rows, f, indent=1)
        return
    if args.production or args.ridge_adjoint:
        prec = {None: None, "fp32": FP32, "fp64": FP64, "fp16": FP16_DEV, "bf16": BF16_DEV}[args.precision]
        if args.production:
            res = production_run(args.production, None if args.steps == 20000 else args.steps, prec, args.chunk)
        else:
            steps = 2500 if args.steps == 20000 else args.steps
            res = ridge_adjoint(scale=args.scale, re=float(args.re) if "," not in args.re else 500.0, steps=steps,
                                avg_steps=args.avg or steps // 4, checkpoints=args.checkpoints, dh=args.dh,
                                precision=FP64 if prec is None else prec)
        print(json.dumps(res))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)
        return
    if args.chaos:
        rows = chaos_study(tuple(float(x) for x in args.re.split(",")), args.steps, args.steps // 2)
        for r in rows:
            print(json.dumps(r), flush=True)
        if args.out:
            with open(args.out, "w") as f:
                json.dump(rows, f, indent=1)
        return
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

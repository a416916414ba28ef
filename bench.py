#!/usr/bin/env python
"""Benchmark of the B200 D3Q19 BGK time step (MLUPS and % of the HBM roofline).

Default workload: the production-size GPU configuration, a 768x384x384
channel with a reticular cylindrical shell (outer D 96, length 256, struts
d=4 at pitch 16 plus diagonals), inlet u=0.05, Re 2000, FP32 populations.
Synthetic inputs: the geometry is voxelised from its seeded analytic
description and the state is a seeded equilibrium (the reference's production
geometry files are unshipped).

One JSON line is printed by rank 0:
  value  - node updates per second (MLUPS) of K time steps with the state
           resident in HBM, timed with CUDA events on the solver's stream;
  e2e    - the same metric through the C ABI with host buffers: upload of the
           haloed state from pinned memory, K eup_step(1) calls each followed
           by the FP64 force read-back, download of the state;
  roofline - the stream-collide kernel's algorithmic bytes per launch (19 reads
           + 19 writes of S-byte populations per node) over its mean launch
           time from CUDA events, against the measured HBM copy bandwidth;
  cpu_baseline - the CPU oracle (restatement of the reference's serial step,
           OpenMP over all host cores) on the same workload;
  precision_forms - (one GPU) the same workload with populations stored as
           FP16 and BF16 deviations: step time, MLUPS, ratio to the FP32 line,
           stream-collide roofline at 76 B/node; and the velocity / C_d error of
           both against an FP64 run on the 256x128x64 cylinder channel;
  adjoint - (one GPU) the 192x96x96 partial-bounce-back channel, 4000 steps:
           checkpointed adjoint time over forward time, FP32 against FP64 gradient.
`--impl reference` times only the CPU oracle (the reference arm); it builds its
input (obstacle mask, seeded initial state) with the oracle alone.
Multi-GPU (torchrun): by default the channel grows with N and is cut into
x-slabs, one per GPU, with the NCCL plane exchange every step (weak scaling);
`--decomp replicas` runs one independent lattice per GPU instead.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PRECISIONS = {"fp32": (0, 4, "f32"), "fp64": (1, 8, "f64"), "fp16": (2, 2, "f16-dev/f32"), "bf16": (3, 2, "bf16-dev/f32")}

# The two benchmark workloads as plain numbers.  The eup arm builds them through
# euplectella_hpc_b200.workloads; the reference arm from these numbers with the oracle
# alone (a CPU test holds the two descriptions equal, mask and initial state included).
#   bc: reference face flags (front, rear, right, left, up, down); svisc = u_in * d / re.
SPECS = {
    "shell": {"name": "reticular_shell_768x384x384_re2000", "lattice": (768, 384, 384), "bc": (5, 4, 3, 3, 3, 3),
              "u_in": 0.05, "re": 2000.0, "d": 96.0, "seed": 2024,
              "body": {"kind": "shell", "x0": 192.0, "length": 256.0, "yc": 192.5, "zc": 192.5, "outer_d": 96.0,
                       "strut_d": 4.0, "pitch": 16.0, "seed": 2024}},
    "cylinder": {"name": "cylinder_256x128x64_re100", "lattice": (256, 128, 64), "bc": (5, 4, 3, 3, 0, 0),
                 "u_in": 0.05, "re": 100.0, "d": 20.0, "seed": 1234,
                 "body": {"kind": "cylinder_z", "xc": 64.0, "yc": 64.0, "r": 10.0}},
}
PERTURBATION = 1e-4


def spec_svisc(spec):
    return spec["u_in"] * spec["d"] / spec["re"]


def config_dict(spec, precision, solid_voxels, world=1):
    """The `config` of the JSON line, the same for both arms."""
    lx, ly, lz = spec["lattice"]
    sbytes = PRECISIONS[precision][1]
    if world > 1:
        return {"workload": f"{spec['name']} x{world} in series", "lattice": [lx * world, ly, lz],
                "nodes": lx * ly * lz * world, "precision": precision, "solid_voxels": solid_voxels * world,
                "bc": list(spec["bc"]), "svisc": spec_svisc(spec), "l2_flush": "inputs larger than L2",
                "parallelism": f"x-slabs x{world}, NCCL plane exchange every step"}
    return {"workload": spec["name"], "lattice": [lx, ly, lz], "nodes": lx * ly * lz, "precision": precision,
            "solid_voxels": solid_voxels, "bc": list(spec["bc"]), "svisc": spec_svisc(spec),
            "l2_flush": f"inputs larger than L2 (lattice {2 * 19 * sbytes * lx * ly * lz / 1e9:.2f} GB >> 126 MB)"}


def reference_input(spec, dtype):
    """Obstacle mask and seeded initial state of a workload, built by the oracle only."""
    from oracle import oracle as O
    lx, ly, lz = spec["lattice"]
    b = spec["body"]
    if b["kind"] == "shell":
        obs = O.voxelise_shell(lx, ly, lz, b["x0"], b["length"], b["yc"], b["zc"], b["outer_d"], b["strut_d"],
                               b["pitch"], b["seed"])
    else:
        obs = O.voxelise_cylinder_z(lx, ly, lz, b["xc"], b["yc"], b["r"])
    state = O.init_perturbed(lx, ly, lz, spec["u_in"], PERTURBATION, spec["seed"], dtype)
    return obs, state


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["eup", "reference"], default="eup")
    ap.add_argument("--workload", choices=["shell", "cylinder"], default="shell")
    ap.add_argument("--precision", choices=list(PRECISIONS), default="fp32")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample length")
    ap.add_argument("--no-extras", action="store_true",
                    help="one GPU: skip the FP16/BF16 and adjoint measurements after the FP32 line")
    ap.add_argument("--decomp", choices=["slabs", "replicas"], default="slabs",
                    help="N > 1: x-slabs of one channel with the plane exchange every step (default), or "
                         "independent replicas")
    return ap.parse_args()


def make_workload(name, precision):
    from euplectella_hpc_b200 import workloads
    if name == "shell":
        return workloads.reticular_shell_channel(precision=precision)
    return workloads.cylinder_channel(precision=precision)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi's start-up (driver queries) stays out of the timed region: wait, at most
        # 3 s, for its first sample
        t0 = time.time()
        while time.time() - t0 < 3.0 and self.proc.poll() is None and os.path.getsize(self.file.name) == 0:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(", ") for r in open(self.file.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < len(self.FIELDS):
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if d.get("hbm_gbs"):
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s)"


def traffic_per_node(prec_name):
    """DRAM bytes per node of one stream-collide launch from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "stream_collide_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(prec_name, {}).get("dram_bytes_per_node")


def cpu_baseline(wl, state, seconds, prec_name):
    """Time the CPU oracle on the same workload, all host cores, about `seconds` of work."""
    from oracle import oracle as O
    c = wl.cfg
    dt = np.float64 if prec_name == "fp64" else np.float32
    a = np.ascontiguousarray(state, dtype=dt)
    p = O.params(c.lx, c.ly, c.lz, c.bc, svisc=c.svisc, u0=c.u0, u_inflow=c.u_inflow, u00=c.u00)
    b = np.empty_like(a)
    t0 = time.perf_counter()
    O.run(p, a, wl.obs, 1, b)
    t1 = time.perf_counter() - t0
    steps = int(max(1, min(200, seconds / max(t1, 1e-6))))
    t0 = time.perf_counter()
    O.run(p, a, wl.obs, steps, b)
    dt_s = time.perf_counter() - t0
    return {"value": wl.nodes * steps / dt_s / 1e6, "unit": "MLUPS", "cores": O.nthreads(), "kind": "port",
            "sample": f"{steps} full time steps of the {wl.name} lattice ({wl.nodes} nodes), "
                      f"{'float' if dt == np.float32 else 'double'} oracle, OpenMP {O.nthreads()} threads"}


def run_reference(args):
    """The reference arm: the CPU oracle (C restatement of the reference's serial step, the
    Fortran reference having no compiler here) on the host cores, on the eup arm's workload,
    with its input built by the oracle alone (no GPU library is loaded)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    from oracle import oracle as O
    spec = SPECS[args.workload]
    dt = np.float64 if args.precision == "fp64" else np.float32
    obs, state = reference_input(spec, dt)
    lx, ly, lz = spec["lattice"]
    nodes = lx * ly * lz
    p = O.params(lx, ly, lz, spec["bc"], svisc=spec_svisc(spec), u_inflow=spec["u_in"])
    b = np.empty_like(state)
    t0 = time.perf_counter()
    O.run(p, state, obs, 1, b)  # first warm-up step, also sizes the sample
    t1 = time.perf_counter() - t0
    budget = 150.0
    warm = max(0, min(args.warmup - 1, int(0.1 * budget / max(t1, 1e-6))))
    O.run(p, state, obs, warm, b)
    steps = int(max(1, min(args.steps, (0.9 * budget) / max(t1, 1e-6))))
    t0 = time.perf_counter()
    O.run(p, state, obs, steps, b)
    dt_s = time.perf_counter() - t0
    v = nodes * steps / dt_s / 1e6
    what = f"the {nodes}-node lattice" if world == 1 else f"one {lx}x{ly}x{lz} x-slab (with its body) of the {world}-slab channel"
    sample = (f"{steps} of {args.steps} requested time steps of {what}, {1 + warm} warm-up; CPU oracle "
              f"(C restatement of the serial reference step; the Fortran reference has no compiler here), "
              f"{'float' if dt == np.float32 else 'double'}, OpenMP {O.nthreads()} threads; input built by the "
              f"oracle (no GPU library loaded)")
    line = {"impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": steps, "warmup": 1 + warm, "ms_per_step": dt_s * 1e3 / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": PRECISIONS[args.precision][2], "data": "synthetic",
            "config": config_dict(spec, args.precision, int(obs.sum()), world),
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": O.nthreads(), "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_eup(args):
    import torch
    import euplectella_hpc_b200 as E

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)

    def barrier():
        if dist is not None:
            dist.barrier()

    prec_code, sbytes, dtype_name = PRECISIONS[args.precision]
    wl = make_workload(args.workload, prec_code)
    wl.cfg.device = local
    c = wl.cfg
    solver = E.Solver(wl.cfg)
    solver.set_obstacles(wl.obs)
    hdt = np.float64 if args.precision == "fp64" else np.float32
    eb = 8 if hdt == np.float64 else 4
    host = torch.empty(solver.shape, dtype=torch.float64 if eb == 8 else torch.float32, pin_memory=True)
    hnp = host.numpy()
    E.lib.eup_init_equilibrium(c.lx, c.ly, c.lz, 0.05, 1e-4, wl.seed, eb, E._ptrs(hnp))
    ptrs = [hnp[q].ctypes.data for q in range(19)]
    state_bytes = hnp.nbytes
    solver.upload_ptrs(ptrs, eb)
    # warm-up through the same path as the timed steps: the step graphs are captured and
    # instantiated here, not inside the timed region
    solver.step(max(args.warmup, 1))
    torch.cuda.synchronize()
    barrier()
    s_solver = torch.cuda.ExternalStream(solver.stream())
    clocks = ClockSampler(local)
    clocks.start()
    # timed region: K time steps (each one CUDA-graph launch of the step's kernels)
    launches0 = solver.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(s_solver)
    solver.step(args.steps)
    ev1.record(s_solver)
    ev1.synchronize()
    launches = solver.launches - launches0
    t_ms = ev0.elapsed_time(ev1)
    # the same K steps again with CUDA events between the phases of every step
    ms = solver.step_profiled(args.steps)  # [bounce+drag, halo planes, stream-collide, total] device ms
    clk = clocks.stop()
    torch.cuda.synchronize()
    barrier()
    if dist is not None:
        t = torch.tensor([t_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    value = world * wl.nodes * args.steps / (t_ms / 1e3) / 1e6
    f_last = solver.forces()

    # roofline of the dominant kernel (stream-collide)
    k_ms = ms[2] / args.steps
    alg_bytes = 2 * 19 * sbytes * wl.nodes
    achieved = alg_bytes / (k_ms / 1e3) / 1e9
    peak, peak_src = measured_peak()
    tpn = traffic_per_node(args.precision)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (tpn * wl.nodes if tpn is not None else None),
            "kernel": "k_stream_collide_scalar" if args.precision == "fp64" else "k_stream_collide_pair",
            "kernel_ms": k_ms, "peak_source": peak_src,
            "phase_ms_per_step": {"bounce_drag": ms[0] / args.steps, "halo_planes": ms[1] / args.steps,
                                  "stream_collide": k_ms, "step_without_graphs": ms[3] / args.steps}}

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        s = torch.cuda.ExternalStream(solver.stream())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier()
        ev0.record(s)
        solver.upload_ptrs(ptrs, eb, itime=0)
        for _ in range(args.steps):
            solver.step(1)
            solver.forces()
        solver.download_ptrs(ptrs, eb)
        ev1.record(s)
        ev1.synchronize()
        e_ms = ev0.elapsed_time(ev1)
        if dist is not None:
            t = torch.tensor([e_ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        e2e = {"value": world * wl.nodes * args.steps / (e_ms / 1e3) / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": (state_bytes + 24 * args.steps) / args.steps,
               "ms_total": e_ms, "path": "eup_upload(pinned) + K x (eup_step(1) + eup_get_forces) + eup_download"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        cpu = cpu_baseline(wl, hnp, args.cpu_seconds, args.precision)

    itime = solver.itime
    solver.close()
    extras = {}
    if world == 1 and not args.no_extras:
        extras["precision_forms"] = precision_forms(args, wl, value, t_ms / args.steps, k_ms, local)
        extras["adjoint"] = adjoint_cost(local)

    if rank == 0:
        config = config_dict(SPECS[args.workload], args.precision, int(wl.obs.sum()))
        if world > 1:
            config["workload"] = f"{wl.name} x{world} replicas"
            config["nodes"] = wl.nodes * world
        line = {"metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype_name, "data": "synthetic", "config": config,
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "roofline": roof, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
                # force on the body after the timed steps from an impulsive start: a check that the
                # state stayed finite, not a drag coefficient of the developed flow
                "state_check": {"fx_after_timed_steps": f_last[0], "itime": itime}}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def _timed_steps(solver, steps, torch):
    """Device ms of `steps` time steps (CUDA events on the solver's stream) and the stream-collide
    ms per step from a profiled pass over the same number of steps."""
    st = torch.cuda.ExternalStream(solver.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    solver.step(steps)
    e1.record(st)
    e1.synchronize()
    ms = solver.step_profiled(steps)
    return e0.elapsed_time(e1) / steps, ms[2] / steps


def precision_forms(args, wl, fp32_mlups, fp32_step_ms, fp32_kernel_ms, device):
    """FP16 and BF16 deviation storage on the bench workload (same box, same process as the FP32
    line), and their accuracy against an FP64 run of the same kernel on the 256x128x64 cylinder
    channel (velocity relative L2 over the fluid after 2000 steps, C_d averaged over the last 500)."""
    import dataclasses as dc

    import torch
    import euplectella_hpc_b200 as E
    from euplectella_hpc_b200 import workloads
    from euplectella_hpc_b200.studies import velocity

    steps = max(100, min(args.steps, 300))
    peak, _ = measured_peak()
    out = {"steps": steps, "warmup": max(args.warmup, 3), "fp32_step_ms": fp32_step_ms,
           "fp32_stream_collide_ms": fp32_kernel_ms}
    for name, code in (("fp16", E.FP16_DEV), ("bf16", E.BF16_DEV)):
        cfg = dc.replace(wl.cfg, precision=code, device=device)
        with E.Solver(cfg) as s:
            s.set_obstacles(wl.obs)
            s.init_state(0.05, 1e-4, wl.seed)
            s.step(max(args.warmup, 3))  # graphs captured outside the timed steps
            step_ms, k_ms = _timed_steps(s, steps, torch)
        mlups = wl.nodes / (step_ms / 1e3) / 1e6
        ach = 2 * 19 * 2 * wl.nodes / (k_ms / 1e3) / 1e9
        out[name] = {"step_ms": step_ms, "mlups": mlups, "over_fp32_mlups": mlups / fp32_mlups,
                     "stream_collide_ms": k_ms, "stream_collide_over_fp32": fp32_kernel_ms / k_ms,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "bytes_per_node": 76}}
    # accuracy on the cylinder channel against FP64
    cyl = workloads.cylinder_channel()
    fluid = cyl.obs == 0
    a0 = cyl.initial_state(np.float64)
    runs = {}
    for name, code in (("fp64", E.FP64), ("fp16", E.FP16_DEV), ("bf16", E.BF16_DEV), ("fp32", E.FP32)):
        with E.Solver(dc.replace(cyl.cfg, precision=code, device=device)) as s:
            s.set_obstacles(cyl.obs)
            s.upload(a0)
            s.step(2000)
            runs[name] = (velocity(s.download(np.float64))[:, fluid], s.cd_series(1501, 500).mean())
    u64, cd64 = runs["fp64"]
    acc = {"workload": cyl.name, "steps": 2000, "cd_window": "steps 1501-2000", "cd_mean_fp64": cd64}
    for name in ("fp32", "fp16", "bf16"):
        u, cd = runs[name]
        acc[name] = {"velocity_rel_l2": float(np.linalg.norm(u - u64) / np.linalg.norm(u64)),
                     "cd_rel_err": abs(cd - cd64) / abs(cd64)}
    out["accuracy_vs_fp64"] = acc
    return out


def adjoint_cost(device):
    """The 192x96x96 partial-bounce-back channel (Re 100, 4000 steps, objective mean C_d over the
    last 1000): adjoint with recomputation from checkpoints over the forward run, against the
    partial-bounce-back forward and against the plain halfway-bounce-back FP32 step on the same
    lattice (body = n_s > 1/2); FP32 against FP64 gradient."""
    import dataclasses as dc

    import torch
    import euplectella_hpc_b200 as E
    from euplectella_hpc_b200 import workloads

    T, A = 4000, 1000
    out = {"workload": "pbb_cylinder_192x96x96_re100", "steps": T, "avg_steps": A}
    grads = {}
    for name, code, dt in (("fp32", E.FP32, np.float32), ("fp64", E.FP64, np.float64)):
        wl = workloads.pbb_cylinder_channel(steps=T, avg_steps=A, precision=code)
        cfg = dc.replace(wl.cfg, device=device)
        a = wl.initial_state(dt)
        with E.Solver(cfg) as s:
            s.set_solid_fraction(wl.ns)
            s.upload(a)
            s.step(3)  # graphs captured outside the timed steps
            fwd_ms = _timed_steps(s, T, torch)[0] * T
        with E.Solver(cfg) as s:  # warm-up: a short adjoint run loads the kernels it uses
            s.set_solid_fraction(wl.ns)
            s.upload(a)
            s.adjoint(64, 16, 8)
        with E.Solver(cfg) as s:
            s.set_solid_fraction(wl.ns)
            s.upload(a)
            J, g, st = s.adjoint(T, A, 64)
        grads[name] = g
        adj_ms = st["forward_ms"] + st["reverse_ms"]
        row = {"objective": J, "pbb_forward_ms": fwd_ms, "adjoint_ms": adj_ms,
               "adjoint_forward_sweep_ms": st["forward_ms"], "adjoint_reverse_ms": st["reverse_ms"],
               "adjoint_over_pbb_forward": adj_ms / fwd_ms, "recomputed_steps": st["recomputed_steps"],
               "stored_states": st["checkpoints"], "repetitions": st["repetitions"],
               "stored_state_bytes": st["state_bytes"]}
        if name == "fp32":
            with E.Solver(cfg) as s:
                s.set_obstacles((wl.ns > 0.5).astype(np.int32))
                s.upload(a)
                s.step(3)
                plain_ms = _timed_steps(s, T, torch)[0] * T
            row["plain_forward_ms"] = plain_ms
            row["adjoint_over_plain_forward"] = adj_ms / plain_ms
        out[name] = row
    out["grad_fp32_vs_fp64_rel_l2"] = float(np.linalg.norm(grads["fp32"] - grads["fp64"]) /
                                            np.linalg.norm(grads["fp64"]))
    return out


def run_slabs(args):
    """N > 1, one process per GPU: a channel N times as long as the single-GPU workload, cut into
    N x-slabs (each holding one copy of the body, so the per-GPU work is the single-GPU
    workload's: weak scaling), stepped with the NCCL plane exchange between the halves of every
    step.  Timed with CUDA events on each slab's stream, max over ranks."""
    import dataclasses as dc

    import torch
    import torch.distributed as dist
    import euplectella_hpc_b200 as E
    from euplectella_hpc_b200.slabs import DistTransport, SlabSolver

    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    prec_code, sbytes, dtype_name = PRECISIONS[args.precision]
    wl = make_workload(args.workload, prec_code)
    gcfg = dc.replace(wl.cfg, lx=wl.cfg.lx * world, device=local)
    slab = SlabSolver(gcfg, rank, world, DistTransport(rank, world))
    assert slab.nx == wl.cfg.lx
    s = slab.solver
    s.set_obstacles(wl.obs)
    s.init_state(0.05, 1e-4, wl.seed + rank)
    slab.step(max(args.warmup, 3))
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = s.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(slab.stream)
    slab.step(args.steps)
    ev1.record(slab.stream)
    ev1.synchronize()
    launches = s.launches - launches0
    t = torch.tensor([ev0.elapsed_time(ev1)], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_ms = float(t.item())
    # stream-collide share: events around the second half of each step (unpack of the received
    # planes, stream-collide, force of the new state)
    ms_end = 0.0
    for _ in range(min(args.steps, 50)):
        slab.begin()
        slab.exchange()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(slab.stream)
        slab.end()
        a1.record(slab.stream)
        a1.synchronize()
        ms_end += a0.elapsed_time(a1)
    clk = clocks.stop()
    k_ms = ms_end / min(args.steps, 50)
    nodes = wl.nodes
    achieved = 2 * 19 * sbytes * nodes / (k_ms / 1e3) / 1e9
    peak, peak_src = measured_peak()
    tpn = traffic_per_node(args.precision)
    value = world * nodes * args.steps / (t_ms / 1e3) / 1e6
    e2e = None
    if not args.no_e2e:
        hdt = torch.float64 if args.precision == "fp64" else torch.float32
        eb = 8 if args.precision == "fp64" else 4
        host = torch.empty(s.shape, dtype=hdt, pin_memory=True)
        hnp = host.numpy()
        E.lib.eup_init_equilibrium(wl.cfg.lx, wl.cfg.ly, wl.cfg.lz, 0.05, 1e-4, wl.seed + rank, eb, E._ptrs(hnp))
        ptrs = [hnp[q].ctypes.data for q in range(19)]
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(slab.stream)
        s.upload_ptrs(ptrs, eb, itime=0)
        for _ in range(args.steps):
            slab.step(1)
            slab.forces()
        s.download_ptrs(ptrs, eb)
        e1.record(slab.stream)
        e1.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], device="cuda")
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e_ms = float(te.item())
        e2e = {"value": world * nodes * args.steps / (e_ms / 1e3) / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": world * hnp.nbytes / args.steps,
               "d2h_bytes_per_step": world * (hnp.nbytes + 24 * args.steps) / args.steps, "ms_total": e_ms,
               "path": "per slab: eup_upload(pinned) + K x (boundaries, NCCL plane exchange, stream, "
                       "all-reduced force) + eup_download"}
    f = slab.forces()
    if rank == 0:
        line = {"metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": dtype_name, "data": "synthetic",
                "config": config_dict(SPECS[args.workload], args.precision, int(wl.obs.sum()), world),
                "parallelism": f"x-slabs x{world}, NCCL plane exchange every step",
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": (tpn * nodes if tpn is not None else None),
                             "kernel": "k_stream_collide_pair (+ plane unpack and force of the step)",
                             "kernel_ms": k_ms, "peak_source": peak_src},
                "e2e": e2e, "cpu_baseline": None, "clocks": clk, "gpu_launches": launches,
                "state_check": {"fx_after_timed_steps": float(f[0]), "itime": s.itime}}
        print(json.dumps(line), flush=True)
    s.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and args.decomp == "slabs":
        return run_slabs(args)
    return run_eup(args)


if __name__ == "__main__":
    sys.exit(main())

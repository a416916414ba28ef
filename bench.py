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
           OpenMP over all host cores) on the same workload.
`--impl reference` times only the CPU oracle (the reference arm).
Multi-GPU (torchrun): one independent lattice per GPU (replicas, weak scaling).
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
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    wl = make_workload(args.workload, PRECISIONS[args.precision][0])
    state = wl.initial_state(np.float64 if args.precision == "fp64" else np.float32)
    from oracle import oracle as O
    c = wl.cfg
    p = O.params(c.lx, c.ly, c.lz, c.bc, svisc=c.svisc, u0=c.u0, u_inflow=c.u_inflow, u00=c.u00)
    b = np.empty_like(state)
    t0 = time.perf_counter()
    O.run(p, state, wl.obs, 1, b)  # first warm-up step, also sizes the sample
    t1 = time.perf_counter() - t0
    budget = 150.0
    warm = max(0, min(args.warmup - 1, int(0.1 * budget / max(t1, 1e-6))))
    O.run(p, state, wl.obs, warm, b)
    steps = int(max(1, min(args.steps, (0.9 * budget) / max(t1, 1e-6))))
    t0 = time.perf_counter()
    O.run(p, state, wl.obs, steps, b)
    dt_s = time.perf_counter() - t0
    v = wl.nodes * steps / dt_s / 1e6
    sample = (f"{steps} of {args.steps} requested time steps (each the full {wl.nodes}-node lattice), "
              f"{1 + warm} warm-up; CPU oracle (C restatement of the serial reference step; the Fortran "
              f"reference has no compiler here), OpenMP {O.nthreads()} threads")
    line = {"impl": "reference", "metric": "MLUPS", "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": steps, "warmup": 1 + warm, "ms_per_step": dt_s * 1e3 / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": PRECISIONS[args.precision][2], "data": "synthetic",
            "config": {"workload": wl.name, "lattice": [c.lx, c.ly, c.lz], "nodes": wl.nodes},
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
    if args.warmup > 0:
        solver.step_profiled(args.warmup)
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
    cd = solver.cd_series(solver.itime, 1)[0]

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

    if rank == 0:
        line = {"metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype_name, "data": "synthetic",
                "config": {"workload": wl.name, "lattice": [c.lx, c.ly, c.lz], "nodes": wl.nodes,
                           "precision": args.precision, "solid_voxels": int(wl.obs.sum()),
                           "bc": list(c.bc), "svisc": c.svisc, "l2_flush": "inputs larger than L2 (lattice "
                           f"{2 * 19 * sbytes * wl.nodes / 1e9:.1f} GB >> 126 MB)",
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "roofline": roof, "e2e": e2e, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches,
                "drag": {"fx": f_last[0], "cd": cd, "itime": solver.itime}}
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


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
        c = wl.cfg
        line = {"metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": dtype_name, "data": "synthetic",
                "config": {"workload": f"{wl.name} x{world} in series", "lattice": [c.lx * world, c.ly, c.lz],
                           "nodes": nodes * world, "precision": args.precision, "bc": list(gcfg.bc),
                           "svisc": c.svisc, "l2_flush": "inputs larger than L2",
                           "parallelism": f"x-slabs x{world}, NCCL plane exchange every step"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": (tpn * nodes if tpn is not None else None),
                             "kernel": "k_stream_collide_pair (+ plane unpack and force of the step)",
                             "kernel_ms": k_ms, "peak_source": peak_src},
                "e2e": e2e, "cpu_baseline": None, "clocks": clk, "gpu_launches": launches,
                "drag": {"fx": float(f[0]), "itime": s.itime}}
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

"""x-slab decomposition on the GPU.  Slabs of one lattice, stepped with the
plane exchange between the halves of each step, must equal the single-lattice
run bit for bit.  Two forms: several slabs in one process (exchange by device
copies), and two processes exchanging through torch.distributed (gloo, host
staging) -- both ranks on the one GPU a test gets, which is fine here because
no kernel waits on another rank: the host orders every exchange."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, M, N = 60, 18, 10


def _case(eup, precision):
    bc = (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    cfg = eup.Config(L, M, N, bc=bc, svisc=0.01, u_inflow=0.05, precision=precision, cd_uref=0.05, cd_length=6,
                     cd_span=N)
    obs = eup.geometry_cylinder_z(L, M, N, 8, 9.5, 3)  # solid columns 5..11, away from every slab face
    return cfg, obs


def _single(eup, cfg, obs, a, steps, dt):
    with eup.Solver(cfg) as s:
        s.set_obstacles(obs)
        s.upload(a)
        s.step(steps)
        return s.download(dt), s.forces()


@pytest.mark.parametrize("split", [False, True], ids=["sequential", "interior_then_faces"])
@pytest.mark.parametrize("prec,world,pack", [("fp32", 3, "view"), ("fp64", 2, "view"), ("fp16", 4, "view"),
                                             ("fp32", 3, "kernel"), ("fp16", 2, "kernel")])
def test_slabs_in_one_process_equal_single_lattice(eup, require_gpu, prec, world, split, pack):
    from euplectella_hpc_b200.slabs import SlabSolver, gather_state, step_in_process
    code, dt = {"fp32": (eup.FP32, np.float32), "fp64": (eup.FP64, np.float64), "fp16": (eup.FP16_DEV, np.float32)}[prec]
    cfg, obs = _case(eup, code)
    a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 5, dt)
    steps = 30
    ref, f_ref = _single(eup, cfg, obs, a, steps, dt)
    slabs = [SlabSolver(cfg, r, world, pack=pack) for r in range(world)]
    try:
        for s in slabs:
            s.set_obstacles(obs)
            s.upload(a)
        step_in_process(slabs, steps, split=split)
        got = gather_state(slabs, dt)
        f = sum(s.solver.forces() for s in slabs)
        assert all(s.solver.itime == steps for s in slabs)
    finally:
        for s in slabs:
            s.solver.close()
    keep = np.ones(got.shape[1:], bool)
    keep[1:-1, 1:-1, 1:-1] = obs == 0
    if prec == "fp16":
        # 16-bit storage keeps deviations in the lattice but f in the FP32 halo, so a pull across
        # a slab face reads the deviation back through f; where that rounding moves a stored
        # deviation by one 16-bit step (2^-5 / 4096 = 7.6e-6 in f for |f - w| < 1/64) the runs
        # part by that quantum: a few quanta at most, almost everywhere none
        d = np.abs(got - ref)[:, keep]
        assert d.max() < 8 * 7.7e-6, d.max()
        assert d.mean() < 2e-6, d.mean()
        np.testing.assert_allclose(f, f_ref, rtol=0, atol=1e-3 * np.abs(f_ref).max())
        return
    for q in range(19):
        bad = (got[q] != ref[q]) & keep
        assert not bad.any(), f"population {q + 1}: {bad.sum()} mismatches, first at {np.argwhere(bad)[0]}"
    np.testing.assert_allclose(f, f_ref, rtol=1e-12, atol=1e-14)


def test_slab_guards(eup, require_gpu):
    from euplectella_hpc_b200.slabs import slab_config
    cfg, obs = _case(eup, eup.FP32)
    c1 = slab_config(cfg, 1, 3)
    with eup.Solver(c1) as s:
        s.upload(eup.init_equilibrium(c1.lx, M, N, 0.05, 0, 1, np.float32))
        with pytest.raises(eup.EupError):
            s.step(1)                      # an x-slab steps only in halves
        with pytest.raises(eup.EupError):
            s.step_stream()                # the boundaries half comes first
        with pytest.raises(eup.EupError):
            s.step_stream_interior()
        s.step_boundaries()
        with pytest.raises(eup.EupError):
            s.step_stream_faces()          # the interior part comes first
        s.step_stream_interior()
        with pytest.raises(eup.EupError):
            s.step_stream()                # the step is half streamed
        with pytest.raises(eup.EupError):
            s.step_boundaries()
        bad = np.zeros((N, M, c1.lx), np.int32)
        bad[3, 4, 0] = 1                   # solid next to the rear exchange face
        with pytest.raises(eup.EupError):
            s.set_obstacles(bad)
        assert s.x_planes_view(0) and s.x_planes_view(1)
    with eup.Solver(slab_config(cfg, 0, 3)) as s:  # first slab: its x = 0 face is the inlet
        assert s.x_planes_view(1)
        with pytest.raises(eup.EupError):
            s.x_planes_view(0)
        with pytest.raises(eup.EupError):
            s.set_x_planes_view(0, s.x_planes_view(1))
        with pytest.raises(eup.EupError):
            s.x_planes_view(2)


def _view_as_planes(v, m, n, side):
    """A plane message in the x-face copy's order (side 1: blocks then rim; side 0: rim then
    blocks) -> (5, n+2, m+2) planes [c, k, j]."""
    out = np.full((5, n + 2, m + 2), np.nan, v.dtype)
    mn, nr = m * n, 5 * (2 * (m + 2) + 2 * n)
    blocks, rim = (v[:5 * mn], v[5 * mn:]) if side else (v[nr:], v[:nr])
    out[:, 1:-1, 1:-1] = blocks.reshape(5, n, m)
    rim = rim.reshape(5, 2 * (m + 2) + 2 * n)
    out[:, 0, :] = rim[:, :m + 2]
    out[:, n + 1, :] = rim[:, m + 2:2 * (m + 2)]
    out[:, 1:-1, 0] = rim[:, 2 * (m + 2):2 * (m + 2) + n]
    out[:, 1:-1, m + 1] = rim[:, 2 * (m + 2) + n:]
    return out


@pytest.mark.parametrize("prec", ["fp32", "fp64", "fp16", "bf16"])
def test_plane_view_equals_pack_kernel(eup, require_gpu, prec):
    """The plane messages read in place from the x-face copy (the stream-collide epilogue's
    face columns, the halo rows packed by step_boundaries) hold, step after step, the values the
    separate pack kernel gathers from the lattice, in the view's order."""
    import torch
    from euplectella_hpc_b200.slabs import SlabSolver, plane_size
    code, dt = {"fp32": (eup.FP32, np.float32), "fp64": (eup.FP64, np.float64), "fp16": (eup.FP16_DEV, np.float32),
                "bf16": (eup.BF16_DEV, np.float32)}[prec]
    tdt = torch.float64 if prec == "fp64" else torch.float32
    cfg, obs = _case(eup, code)
    a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 5, dt)
    s = SlabSolver(cfg, 1, 3)  # the middle slab: both x faces exchange
    n = plane_size(cfg)
    try:
        s.set_obstacles(obs)
        s.upload(a)
        for _ in range(6):
            s.begin()
            for side, key in ((0, "send_l"), (1, "send_r")):
                packed = torch.empty(n, dtype=tdt, device="cuda")
                s.solver.get_x_planes(side, packed.data_ptr())
                s.solver.synchronize()
                want = packed.cpu().numpy().reshape(5, N + 2, M + 2)
                got = _view_as_planes(s.buf[key].cpu().numpy(), M, N, side)
                assert np.array_equal(got, want), (side, np.argwhere(got != want)[:4])
                assert np.isfinite(got).all()
            # close the slab on itself (finite, consistent planes) and finish the step
            s.buf["recv_l"].copy_(s.buf["send_r"])
            s.buf["recv_r"].copy_(s.buf["send_l"])
            torch.cuda.synchronize()
            s.end()
    finally:
        s.solver.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_worker(rank, world, port, prec, steps, out_dir):
    import torch
    import torch.distributed as dist
    import euplectella_hpc_b200 as eup
    from euplectella_hpc_b200.slabs import DistTransport, SlabSolver
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        code, dt = (eup.FP32, np.float32) if prec == "fp32" else (eup.FP64, np.float64)
        cfg, obs = _case(eup, code)
        a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 5, dt)
        s = SlabSolver(cfg, rank, world, DistTransport(rank, world))
        s.set_obstacles(obs)
        s.upload(a)
        s.step(steps)
        f = s.forces()
        np.save(os.path.join(out_dir, f"slab{rank}.npy"), s.solver.download(dt))
        np.save(os.path.join(out_dir, f"force{rank}.npy"), f)
        s.solver.close()
    finally:
        dist.destroy_process_group()


def test_two_ranks_through_torch_distributed(eup, require_gpu, tmp_path):
    import torch.multiprocessing as mp
    from euplectella_hpc_b200.slabs import partition
    world, steps = 2, 20
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, world, port, "fp32", steps, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    cfg, obs = _case(eup, eup.FP32)
    a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 5, np.float32)
    ref, f_ref = _single(eup, cfg, obs, a, steps, np.float32)
    for r, (x0, nx) in enumerate(partition(L, world)):
        loc = np.load(tmp_path / f"slab{r}.npy")
        fl = obs[:, :, x0 - 1:x0 - 1 + nx] == 0
        for q in range(19):
            got, want = loc[q][1:-1, 1:-1, 1:-1], ref[q][1:-1, 1:-1, x0:x0 + nx]
            assert np.array_equal(got[fl], want[fl]), (r, q)
        np.testing.assert_allclose(np.load(tmp_path / f"force{r}.npy"), f_ref, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("prec,l", [("fp32", 60), ("fp32", 61), ("fp32", 2), ("fp64", 40), ("fp16", 60), ("bf16", 33)])
def test_split_stream_equals_whole_step(eup, require_gpu, prec, l):
    """boundaries + interior columns + face columns gives eup_step's bits (two-node kernel for
    even l, one-node for odd l and FP64; l = 2 has a single pair holding both face columns)."""
    code, dt = {"fp32": (eup.FP32, np.float32), "fp64": (eup.FP64, np.float64), "fp16": (eup.FP16_DEV, np.float32),
                "bf16": (eup.BF16_DEV, np.float32)}[prec]
    bc = (eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC)
    cfg = eup.Config(l, M, N, bc=bc, svisc=0.01, u_inflow=0.05, precision=code)
    obs = eup.geometry_cylinder_z(l, M, N, l / 3, 9.5, 2.5) if l > 8 else np.zeros((N, M, l), np.int32)
    a = eup.init_equilibrium(l, M, N, 0.05, 1e-3, 8, dt)
    out = []
    for split in (False, True):
        with eup.Solver(cfg) as s:
            s.set_obstacles(obs)
            s.upload(a)
            for _ in range(12):
                if split:
                    s.step_boundaries()
                    s.step_stream_interior()
                    s.step_stream_faces()
                else:
                    s.step(1)
            out.append((s.download(dt), s.force_series(0, 13), s.itime))
    assert out[0][2] == out[1][2] == 12
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


class _LocalTransport:
    """Stands in for NCCL between slabs of one process: 'sends' are device copies from the
    neighbour's buffers, issued on the caller's current stream (the exchange stream), after a
    device synchronisation so that every slab's pack has finished."""
    nccl = True

    def __init__(self, slabs, rank):
        self.slabs, self.rank = slabs, rank

    def exchange(self, send_l, send_r, recv_l, recv_r):
        import torch
        torch.cuda.synchronize()
        if self.rank > 0:
            recv_l.copy_(self.slabs[self.rank - 1].buf["send_r"])
        if self.rank < len(self.slabs) - 1:
            recv_r.copy_(self.slabs[self.rank + 1].buf["send_l"])


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_overlapped_exchange_path(eup, require_gpu, prec):
    """SlabSolver.exchange_overlapped (the NCCL step: packed-event wait on the high-priority
    exchange stream, interior stream-collide meanwhile, arrival-event wait, face columns) with
    the transport replaced by device copies: equal to the single lattice bit for bit."""
    from euplectella_hpc_b200.slabs import SlabSolver, gather_state
    code, dt = (eup.FP32, np.float32) if prec == "fp32" else (eup.FP64, np.float64)
    cfg, obs = _case(eup, code)
    a = eup.init_equilibrium(L, M, N, 0.05, 1e-3, 5, dt)
    steps, world = 25, 3
    ref, f_ref = _single(eup, cfg, obs, a, steps, dt)
    slabs = [SlabSolver(cfg, r, world) for r in range(world)]
    try:
        for r, s in enumerate(slabs):
            s.transport = _LocalTransport(slabs, r)
            s.set_obstacles(obs)
            s.upload(a)
        for _ in range(steps):
            for s in slabs:
                s.begin()
            for s in slabs:
                s.exchange_overlapped()
            for s in slabs:
                s.end_faces()
        got = gather_state(slabs, dt)
        f = sum(s.solver.forces() for s in slabs)
    finally:
        for s in slabs:
            s.solver.close()
    keep = np.ones(got.shape[1:], bool)
    keep[1:-1, 1:-1, 1:-1] = obs == 0
    for q in range(19):
        bad = (got[q] != ref[q]) & keep
        assert not bad.any(), f"population {q + 1}: {bad.sum()} mismatches"
    np.testing.assert_allclose(f, f_ref, rtol=1e-12, atol=1e-14)

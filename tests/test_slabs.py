"""x-slab decomposition, host side: the partition, the per-slab configuration
and slicing, and the plane exchange between two gloo ranks on the CPU (the
transport the GPU run uses, with host tensors standing in for the planes)."""
import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_column_once(eup):
    from euplectella_hpc_b200.slabs import partition
    for lx, world in ((768, 1), (768, 2), (1024, 8), (101, 4), (9, 4)):
        parts = partition(lx, world)
        assert len(parts) == world
        cols = [x for x0, nx in parts for x in range(x0, x0 + nx)]
        assert cols == list(range(1, lx + 1))
        widths = [nx for _, nx in parts]
        assert max(widths) - min(widths) <= 1
    with pytest.raises(ValueError):
        partition(7, 4)


def test_slab_config_flags_and_slicing(eup):
    from euplectella_hpc_b200.slabs import partition, slab_config, slab_obstacles, slab_state
    cfg = eup.Config(40, 12, 6, bc=(eup.OUTFLOW, eup.INFLOW, eup.FREESLIP, eup.FREESLIP, eup.PERIODIC, eup.PERIODIC))
    flags = [slab_config(cfg, r, 3).bc[:2] for r in range(3)]
    assert flags == [(eup.EXCHANGE, eup.INFLOW), (eup.EXCHANGE, eup.EXCHANGE), (eup.OUTFLOW, eup.EXCHANGE)]
    assert sum(slab_config(cfg, r, 3).lx for r in range(3)) == 40
    assert slab_config(cfg, 1, 3).bc[2:] == cfg.bc[2:]
    with pytest.raises(ValueError):
        slab_config(eup.Config(40, 12, 6, bc=(0, 0, 3, 3, 0, 0)), 0, 2)
    rng = np.random.default_rng(0)
    pops = rng.standard_normal((19, 8, 14, 42)).astype(np.float32)
    obs = rng.integers(0, 2, (6, 12, 40)).astype(np.int32)
    for x0, nx in partition(40, 3):
        st = slab_state(pops, x0, nx)
        assert st.shape == (19, 8, 14, nx + 2)
        assert np.array_equal(st[:, :, :, 1:-1], pops[:, :, :, x0:x0 + nx])   # interior columns
        assert np.array_equal(st[:, :, :, 0], pops[:, :, :, x0 - 1])          # left halo = previous column
        assert np.array_equal(slab_obstacles(obs, x0, nx), obs[:, :, x0 - 1:x0 - 1 + nx])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from euplectella_hpc_b200.slabs import DistTransport
        t = DistTransport(rank, world)
        n = 7
        send_l = torch.full((n,), 100.0 * rank + 1)   # to rank-1
        send_r = torch.full((n,), 100.0 * rank + 2)   # to rank+1
        recv_l, recv_r = torch.zeros(n), torch.zeros(n)
        t.exchange(send_l, send_r, recv_l, recv_r)
        s = t.allreduce_sum(torch.tensor([float(rank + 1)], dtype=torch.float64))
        q.put((rank, recv_l[0].item(), recv_r[0].item(), s.item(), t.nccl))
    finally:
        dist.destroy_process_group()


def test_plane_exchange_between_gloo_ranks(eup):
    import torch.multiprocessing as mp
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got_l, got_r, total, nccl in res:
        # my left buffer holds the left neighbour's right-going plane, and vice versa
        assert got_l == (100.0 * (rank - 1) + 2 if rank > 0 else 0.0)
        assert got_r == (100.0 * (rank + 1) + 1 if rank < world - 1 else 0.0)
        assert total == 6.0 and not nccl

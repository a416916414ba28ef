"""x-slab decomposition of one lattice over several GPUs (one process per GPU).

The global lattice lx x ly x lz is cut along x into `world` slabs of nearly
equal width; slab r holds nodes x0_r .. x0_r + nx_r - 1 on its own GPU.  The
faces between slabs are flagged EXCHANGE: each step runs

    bounce-back + halo planes          eup_step_boundaries   (every slab; with
                                         an exchange face it also packs the halo
                                         rows of the outgoing plane messages)
    stream-collide of x = 2..l-1       eup_step_stream_interior
      meanwhile send/recv to the       torch.distributed (NCCL: device buffers
      neighbours                       on a high-priority stream, ordered by
                                       events; gloo: staged through host memory)
    unpack into the x halo             eup_set_x_planes_view
    stream-collide of x = 1 and l      eup_step_stream_faces

The messages are sent straight from the handle's x-face copy
(eup_get_x_planes_view): the stream-collide kernel writes the face columns'
populations there in its epilogue, so no kernel packs the planes
(pack="kernel" selects the separate pack kernel, eup_get_x_planes, instead).

Only 5 of the 19 populations cross a face ((ly+2)(lz+2) values each, the y/z
halo rows included, so corner pulls see this step's y/z boundary values): the
+x face carries a01..a05, the -x face a10..a14 (the same populations the
reference packs in CODE/SRC/bcond.comm.packed.F90:203-286).  Because the planes
move after the halo kernels, an FP32 or FP64 slab run equals the single-lattice
run bit for bit; the one condition is that no solid voxel sits on a column next
to an exchange face (its bounce-back would read the neighbour's state of the
previous step), which eup_set_obstacles rejects.  With 16-bit storage the
planes travel as f in FP32 (the halo's type) while the lattice holds 16-bit
deviations, so a pull across a face sees the deviation rounded through f: the
run agrees with the single lattice to FP32 rounding of f instead.  The global x faces keep
their own flags (inflow/outflow/walls); a periodic x axis is not offered across
slabs.  Forces and monitor sums are per slab; their sum is the lattice's.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import EXCHANGE, FP64, PERIODIC, Config, Solver

PLANE_POPS = 5


def partition(lx: int, world: int) -> list[tuple[int, int]]:
    """(x0, nx) per rank: 1-based first column and width, widths differing by at most one."""
    if world < 1 or lx < 2 * world:
        raise ValueError(f"cannot cut {lx} columns into {world} slabs of at least 2")
    base, extra = divmod(lx, world)
    out, x0 = [], 1
    for r in range(world):
        nx = base + (1 if r < extra else 0)
        out.append((x0, nx))
        x0 += nx
    return out


def slab_config(cfg: Config, rank: int, world: int) -> Config:
    """Configuration of slab `rank`: its width, EXCHANGE on the faces shared with a neighbour."""
    if world > 1 and cfg.bc[0] == PERIODIC and cfg.bc[1] == PERIODIC:
        raise ValueError("a periodic x axis is not offered across x-slabs")
    x0, nx = partition(cfg.lx, world)[rank]
    bc = list(cfg.bc)
    if rank < world - 1:
        bc[0] = EXCHANGE  # front: x = nx faces the next slab
    if rank > 0:
        bc[1] = EXCHANGE  # rear: x = 1 faces the previous slab
    return dataclasses.replace(cfg, lx=nx, bc=tuple(bc))


def slab_obstacles(obs: np.ndarray, x0: int, nx: int) -> np.ndarray:
    """Columns x0 .. x0+nx-1 of obs(1:l,1:m,1:n) (shape (n, m, l))."""
    return np.ascontiguousarray(obs[:, :, x0 - 1:x0 - 1 + nx])


def slab_state(pops: np.ndarray, x0: int, nx: int) -> np.ndarray:
    """The haloed state of the slab: global haloed columns x0-1 .. x0+nx (local 0 .. nx+1)."""
    return np.ascontiguousarray(pops[:, :, :, x0 - 1:x0 + nx + 1])


def plane_size(cfg: Config) -> int:
    return PLANE_POPS * (cfg.ly + 2) * (cfg.lz + 2)


class _DeviceArray:
    """A device address seen by torch as a 1-D tensor (CUDA array interface), no copy."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "strides": None, "version": 2}


class DistTransport:
    """Moves the face planes between neighbouring ranks with torch.distributed point-to-point
    operations.  NCCL: the buffers live on the GPU and the operations are ordered on the
    solver's stream.  gloo: device buffers are staged through host memory."""

    def __init__(self, rank: int, world: int, group=None):
        import torch.distributed as dist
        self.dist, self.rank, self.world, self.group = dist, rank, world, group
        self.nccl = dist.get_backend(group) == "nccl"

    def exchange(self, send_left, send_right, recv_left, recv_right):
        """send_left -> rank-1 (its recv_right), send_right -> rank+1 (its recv_left)."""
        ops = []
        P2P = self.dist.P2POp
        if self.rank > 0:
            ops.append(P2P(self.dist.isend, send_left, self.rank - 1, self.group))
            ops.append(P2P(self.dist.irecv, recv_left, self.rank - 1, self.group))
        if self.rank < self.world - 1:
            ops.append(P2P(self.dist.isend, send_right, self.rank + 1, self.group))
            ops.append(P2P(self.dist.irecv, recv_right, self.rank + 1, self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce_sum(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t


class SlabSolver:
    """Slab `rank` of a lattice cut along x, on the current process's GPU."""

    def __init__(self, cfg: Config, rank: int, world: int, transport=None, pack: str = "view"):
        import torch
        if pack not in ("view", "kernel"):
            raise ValueError("pack is 'view' or 'kernel'")
        self.torch = torch
        self.gcfg, self.rank, self.world = cfg, rank, world
        self.x0, self.nx = partition(cfg.lx, world)[rank]
        self.cfg = slab_config(cfg, rank, world)
        self.solver = Solver(self.cfg)
        self.transport = transport
        self.pack = pack
        dt = torch.float64 if cfg.precision == FP64 else torch.float32
        dev = torch.device("cuda", cfg.device)
        n = plane_size(cfg)
        self.buf = {k: torch.zeros(n, dtype=dt, device=dev) for k in ("send_l", "send_r", "recv_l", "recv_r")}
        if pack == "view":  # send straight from the x-face copy: these tensors alias the handle's memory
            ts = "<f8" if dt == torch.float64 else "<f4"
            for side, key, on in ((0, "send_l", self.has_left), (1, "send_r", self.has_right)):
                if on:
                    self.buf[key] = torch.as_tensor(_DeviceArray(self.solver.x_planes_view(side), n, ts), device=dev)
        staged = transport is not None and not getattr(transport, "nccl", True)
        self.host = {k: torch.zeros(n, dtype=dt, pin_memory=True) for k in self.buf} if staged else None
        self.stream = torch.cuda.ExternalStream(self.solver.stream())
        # the exchange runs beside the interior stream-collide; at high priority its kernels
        # take SMs as the interior blocks retire instead of queueing behind all of them
        self.xstream = torch.cuda.Stream(device=dev, priority=-1)

    # ---- set-up (from the global arrays) ----
    def set_obstacles(self, obs_global: np.ndarray):
        self.solver.set_obstacles(slab_obstacles(obs_global, self.x0, self.nx))

    def build_obstacles(self, geom):
        """Voxelises the global shape `geom` (an eup_geometry in global coordinates) on this
        slab's GPU: the slab's block is the shape shifted by x0 - 1, as the reference offsets a
        block by mpicoords * l (CODE/SRC/build.obs.F90:233-235)."""
        self.solver.build_obstacles(geom.shifted((geom.offset[0] + self.x0 - 1, geom.offset[1], geom.offset[2])))

    def upload(self, pops_global: np.ndarray, itime: int = 0):
        self.solver.upload(slab_state(pops_global, self.x0, self.nx), itime)

    @property
    def has_left(self):
        return self.rank > 0

    @property
    def has_right(self):
        return self.rank < self.world - 1

    # ---- one step in halves, for callers that interleave several slabs ----
    def begin(self):
        self.solver.step_boundaries()
        if self.pack == "kernel":
            if self.has_left:
                self.solver.get_x_planes(0, self.buf["send_l"].data_ptr())
            if self.has_right:
                self.solver.get_x_planes(1, self.buf["send_r"].data_ptr())

    def _unpack(self):
        unpack = self.solver.set_x_planes_view if self.pack == "view" else self.solver.set_x_planes
        if self.has_left:
            unpack(0, self.buf["recv_l"].data_ptr())
        if self.has_right:
            unpack(1, self.buf["recv_r"].data_ptr())

    def end(self):
        self._unpack()
        self.solver.step_stream()

    def end_faces(self):
        """After step_stream_interior and the exchange: unpack, then the x = 1 and x = l columns."""
        self._unpack()
        self.solver.step_stream_faces()

    def exchange(self):
        """Move this step's planes to and from the neighbour ranks."""
        b = self.buf
        if self.world == 1:
            return
        if self.host is None:  # NCCL: device buffers, ordered on the solver's stream
            with self.torch.cuda.stream(self.stream):
                self.transport.exchange(b["send_l"], b["send_r"], b["recv_l"], b["recv_r"])
        else:  # host-staged transport (gloo)
            self.solver.synchronize()
            h = self.host
            for k in ("send_l", "send_r"):
                h[k].copy_(b[k])
            self.transport.exchange(h["send_l"], h["send_r"], h["recv_l"], h["recv_r"])
            for k in ("recv_l", "recv_r"):
                b[k].copy_(h[k])
            self.torch.cuda.synchronize()

    def exchange_overlapped(self):
        """NCCL exchange on the high-priority stream while the solver's stream runs the interior
        stream-collide: the exchange waits for the outgoing planes, the face columns for the
        received ones."""
        torch, b = self.torch, self.buf
        packed = torch.cuda.Event()
        packed.record(self.stream)
        self.solver.step_stream_interior()
        with torch.cuda.stream(self.xstream):
            self.xstream.wait_event(packed)
            self.transport.exchange(b["send_l"], b["send_r"], b["recv_l"], b["recv_r"])
            arrived = torch.cuda.Event()
            arrived.record(self.xstream)
        self.stream.wait_event(arrived)

    def step(self, nsteps: int = 1, overlap: bool = True):
        """nsteps time steps of this slab, exchanging with the neighbour ranks every step; with
        NCCL the exchange overlaps the interior stream-collide (overlap=False: in sequence)."""
        if self.world > 1 and self.transport is None:
            raise ValueError("a slab with neighbours needs a transport (or step_in_process)")
        split = overlap and self.world > 1 and self.host is None
        for _ in range(nsteps):
            self.begin()
            if split:
                self.exchange_overlapped()
                self.end_faces()
            else:
                self.exchange()
                self.end()

    def forces(self) -> np.ndarray:
        """The lattice's momentum-exchange force: the sum over the slabs."""
        f = self.torch.tensor(self.solver.forces(), dtype=self.torch.float64)
        if self.transport is not None:
            if getattr(self.transport, "nccl", False):
                f = f.cuda()
            f = self.transport.allreduce_sum(f)
        return f.cpu().numpy()


def step_in_process(slabs: list[SlabSolver], nsteps: int = 1, split: bool = False):
    """Steps slabs that share one process (and possibly one GPU): the plane exchange is a
    device copy between the slabs' buffers, between the two halves of every slab's step
    (split=True: the interior stream-collide is enqueued before the copy, the face columns
    after it, as the overlapped NCCL step does)."""
    for _ in range(nsteps):
        for s in slabs:
            s.begin()
            if split:
                s.solver.step_stream_interior()
        for s in slabs:
            s.solver.synchronize()
        for r, s in enumerate(slabs):
            if s.has_left:
                s.buf["recv_l"].copy_(slabs[r - 1].buf["send_r"])
            if s.has_right:
                s.buf["recv_r"].copy_(slabs[r + 1].buf["send_l"])
        slabs[0].torch.cuda.synchronize()
        for s in slabs:
            if split:
                s.end_faces()
            else:
                s.end()


def gather_state(slabs: list[SlabSolver], dtype=np.float32) -> np.ndarray:
    """The global haloed state assembled from in-process slabs (interior columns from each slab,
    the global x halo planes from the first and last)."""
    g = slabs[0].gcfg
    out = np.zeros((19, g.lz + 2, g.ly + 2, g.lx + 2), dtype=dtype)
    for s in slabs:
        loc = s.solver.download(dtype)
        out[:, :, :, s.x0:s.x0 + s.nx] = loc[:, :, :, 1:s.nx + 1]
        if s.rank == 0:
            out[:, :, :, 0] = loc[:, :, :, 0]
        if s.rank == len(slabs) - 1:
            out[:, :, :, -1] = loc[:, :, :, -1]
    return out

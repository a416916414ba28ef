"""B200-native D3Q19 BGK lattice-Boltzmann time step for Euplectella_HPC.

The product is the sm_100a shared library `_lib/libeup.so` with the C ABI of
`include/eup.h`; this module is a thin ctypes mirror of that ABI used by the
tests and the benchmark.  It never falls back to a CPU path: when the library
is missing, importing raises, and every call that needs a GPU reports the
library's error.

Array conventions follow the reference (giacomofalcucci/Euplectella_HPC):
populations are one numpy array of shape (19, n+2, m+2, l+2) -- the Fortran
arrays a01..a19(0:l+1,0:m+1,0:n+1) of CODE/SRC/alloca.F90:94-132 stacked, last
axis fastest -- and the solid mask is obs with shape (n, m, l), 1 = solid.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libeup.so")

# Boundary flag codes (CODE/SRC/build.bcond.F90:11-17) and face order.
PERIODIC, NOSLIP, LID, FREESLIP, INFLOW, OUTFLOW, EXCHANGE = range(7)
FRONT, REAR, RIGHT, LEFT, UP, DOWN = range(6)
# Precision modes.
FP32, FP64, FP16_DEV, BF16_DEV = range(4)

STATUS = {0: "EUP_OK", 1: "EUP_ERR_INVALID_ARG", 2: "EUP_ERR_CUDA", 3: "EUP_ERR_OOM", 4: "EUP_ERR_DIVERGED",
          5: "EUP_ERR_UNSUPPORTED", 6: "EUP_ERR_IO", 7: "EUP_ERR_NO_DEVICE"}

EXPORTED = [
    "eup_abi_version", "eup_device_count", "eup_create", "eup_destroy", "eup_last_error", "eup_set_obstacles",
    "eup_upload", "eup_download", "eup_step", "eup_step_profiled", "eup_synchronize", "eup_get_stream", "eup_get_launch_count",
    "eup_get_itime", "eup_get_forces", "eup_get_force_series", "eup_get_cd_series", "eup_get_monitor",
    "eup_get_probes", "eup_get_links", "eup_get_boundary_solid", "eup_read_obs_file", "eup_write_obs_file",
    "eup_read_raw_state", "eup_write_raw_state", "eup_init_equilibrium", "eup_geometry_cylinder_z",
    "eup_geometry_reticular_shell", "eup_mem_force_noalloc", "eup_set_solid_fraction", "eup_adjoint_run",
    "eup_geometry_ridged_shell", "eup_get_region_sums", "eup_init_state", "eup_get_line", "eup_get_plane_means",
    "eup_get_cv_drag", "eup_save_state", "eup_restore_state", "eup_step_boundaries", "eup_step_stream",
    "eup_get_x_planes", "eup_set_x_planes", "eup_geometry_reference", "eup_voxelise", "eup_build_obstacles",
    "eup_get_obstacles", "eup_write_obstacles", "eup_step_stream_interior", "eup_step_stream_faces",
    "eup_init_reference", "eup_adjoint_plan", "eup_get_x_planes_view", "eup_set_x_planes_view",
]


class EupError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class CConfig(ctypes.Structure):
    _fields_ = [
        ("lx", ctypes.c_int32), ("ly", ctypes.c_int32), ("lz", ctypes.c_int32),
        ("bc", ctypes.c_int32 * 6),
        ("svisc", ctypes.c_double), ("u0", ctypes.c_double), ("u_inflow", ctypes.c_double),
        ("u00", ctypes.c_double),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
        ("dev_scale", ctypes.c_double),
        ("cd_rho0", ctypes.c_double), ("cd_uref", ctypes.c_double), ("cd_length", ctypes.c_double),
        ("cd_span", ctypes.c_double),
        ("series_capacity", ctypes.c_int64),
    ]


# Voxel shapes of eup_geometry and the variant bits of eup_geometry_reference.
GEOM_NONE, GEOM_REF_SPHERE, GEOM_REF_COLUMN, GEOM_CYLINDER_Z, GEOM_RETICULAR_SHELL, GEOM_RIDGED_SHELL = range(6)
GEOM_VARIANT_CYLINDER_INF, GEOM_VARIANT_TEST1 = 1, 2


class Geometry(ctypes.Structure):
    """eup_geometry: a voxel shape in global node coordinates (global index = local + offset)."""
    _fields_ = [
        ("kind", ctypes.c_int32), ("offset", ctypes.c_int32 * 3),
        ("center", ctypes.c_int32 * 3), ("kstop", ctypes.c_int32), ("r2_lo", ctypes.c_int64), ("r2_hi", ctypes.c_int64),
        ("xc", ctypes.c_double), ("yc", ctypes.c_double), ("zc", ctypes.c_double), ("radius", ctypes.c_double),
        ("x0", ctypes.c_double), ("length", ctypes.c_double), ("outer_d", ctypes.c_double),
        ("strut_d", ctypes.c_double), ("pitch", ctypes.c_double),
        ("ridge_h", ctypes.c_double), ("ridge_t", ctypes.c_double), ("cap_t", ctypes.c_double),
        ("pore_d", ctypes.c_double), ("seed", ctypes.c_uint64),
    ]

    def shifted(self, offset) -> "Geometry":
        """A copy with another offset (an x-slab's x0 - 1, or the reference's mpicoords * local size)."""
        g = Geometry.from_buffer_copy(self)
        g.offset[:] = [int(v) for v in offset]
        return g

    @staticmethod
    def cylinder_z(xc, yc, r) -> "Geometry":
        g = Geometry(kind=GEOM_CYLINDER_Z)
        g.xc, g.yc, g.radius = float(xc), float(yc), float(r)
        return g

    @staticmethod
    def reticular_shell(x0, length, yc, zc, outer_d, strut_d, pitch, seed) -> "Geometry":
        g = Geometry(kind=GEOM_RETICULAR_SHELL)
        g.x0, g.length, g.yc, g.zc = float(x0), float(length), float(yc), float(zc)
        g.outer_d, g.strut_d, g.pitch, g.seed = float(outer_d), float(strut_d), float(pitch), int(seed)
        return g

    @staticmethod
    def ridged_shell(x0, length, yc, zc, outer_d, strut_d, pitch, ridge_h, ridge_t, cap_t, pore_d, seed) -> "Geometry":
        g = Geometry.reticular_shell(x0, length, yc, zc, outer_d, strut_d, pitch, seed)
        g.kind = GEOM_RIDGED_SHELL
        g.ridge_h, g.ridge_t, g.cap_t, g.pore_d = float(ridge_h), float(ridge_t), float(cap_t), float(pore_d)
        return g


class AdjointConfig(ctypes.Structure):
    _fields_ = [("nsteps", ctypes.c_int32), ("avg_steps", ctypes.c_int32), ("checkpoints", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python euplectella_hpc_b200/build.py` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P19 = ctypes.c_void_p * 19
    sig = {
        "eup_abi_version": ([], i32), "eup_device_count": ([], i32),
        "eup_create": ([ctypes.POINTER(CConfig), ctypes.POINTER(vp)], ctypes.c_int),
        "eup_destroy": ([vp], ctypes.c_int), "eup_last_error": ([vp], ctypes.c_char_p),
        "eup_set_obstacles": ([vp, vp], ctypes.c_int),
        "eup_upload": ([vp, P19, i32, i64], ctypes.c_int), "eup_download": ([vp, P19, i32], ctypes.c_int),
        "eup_step": ([vp, i32], ctypes.c_int), "eup_step_profiled": ([vp, i32, vp], ctypes.c_int),
        "eup_synchronize": ([vp], ctypes.c_int), "eup_get_stream": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "eup_get_launch_count": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_get_itime": ([vp, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_get_forces": ([vp, vp], ctypes.c_int),
        "eup_get_force_series": ([vp, i64, i32, vp], ctypes.c_int),
        "eup_get_cd_series": ([vp, i64, i32, vp], ctypes.c_int),
        "eup_get_monitor": ([vp, vp], ctypes.c_int), "eup_get_probes": ([vp, i32, vp, vp], ctypes.c_int),
        "eup_get_links": ([vp, vp], ctypes.c_int),
        "eup_get_boundary_solid": ([vp, vp, i64, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_read_obs_file": ([ctypes.c_char_p, i32, i32, i32, vp, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_write_obs_file": ([ctypes.c_char_p, i32, i32, i32, vp], ctypes.c_int),
        "eup_read_raw_state": ([ctypes.c_char_p, i32, i32, i32, i32, P19, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_write_raw_state": ([ctypes.c_char_p, i32, i32, i32, i32, P19, i64], ctypes.c_int),
        "eup_init_equilibrium": ([i32, i32, i32, dbl, dbl, ctypes.c_uint64, i32, P19], ctypes.c_int),
        "eup_geometry_cylinder_z": ([i32, i32, i32, dbl, dbl, dbl, vp], ctypes.c_int),
        "eup_geometry_reticular_shell": ([i32, i32, i32, dbl, dbl, dbl, dbl, dbl, dbl, dbl, ctypes.c_uint64, vp],
                                         ctypes.c_int),
        "eup_mem_force_noalloc": ([i32, i32, i32, ctypes.c_int32 * 6, P19, i32, vp, vp, vp], ctypes.c_int),
        "eup_adjoint_plan": ([i32, i32, vp, vp, vp], ctypes.c_int),
        "eup_set_solid_fraction": ([vp, vp], ctypes.c_int),
        "eup_geometry_ridged_shell": ([i32, i32, i32] + [dbl] * 12 + [ctypes.c_uint64, vp, vp], ctypes.c_int),
        "eup_get_region_sums": ([vp, vp, vp], ctypes.c_int),
        "eup_init_state": ([vp, dbl, dbl, ctypes.c_uint64, i64], ctypes.c_int),
        "eup_get_line": ([vp, i32, i32, i32, vp], ctypes.c_int),
        "eup_get_plane_means": ([vp, i32, vp], ctypes.c_int),
        "eup_get_cv_drag": ([vp, vp, vp], ctypes.c_int),
        "eup_save_state": ([vp, ctypes.c_char_p, i32], ctypes.c_int),
        "eup_step_boundaries": ([vp], ctypes.c_int), "eup_step_stream": ([vp], ctypes.c_int),
        "eup_get_x_planes": ([vp, i32, vp], ctypes.c_int), "eup_set_x_planes": ([vp, i32, vp], ctypes.c_int),
        "eup_get_x_planes_view": ([vp, i32, ctypes.POINTER(vp)], ctypes.c_int),
        "eup_set_x_planes_view": ([vp, i32, vp], ctypes.c_int),
        "eup_restore_state": ([vp, ctypes.c_char_p, i32], ctypes.c_int),
        "eup_adjoint_run": ([vp, ctypes.POINTER(AdjointConfig), ctypes.POINTER(dbl), vp, vp], ctypes.c_int),
        "eup_geometry_reference": ([i32, i32, i32, i32, i32, ctypes.POINTER(Geometry)], ctypes.c_int),
        "eup_voxelise": ([ctypes.POINTER(Geometry), i32, i32, i32, vp], ctypes.c_int),
        "eup_build_obstacles": ([vp, ctypes.POINTER(Geometry)], ctypes.c_int),
        "eup_get_obstacles": ([vp, vp, ctypes.POINTER(i64)], ctypes.c_int),
        "eup_write_obstacles": ([vp, ctypes.c_char_p], ctypes.c_int),
        "eup_step_stream_interior": ([vp], ctypes.c_int), "eup_step_stream_faces": ([vp], ctypes.c_int),
        "eup_init_reference": ([i32, i32, i32, i32, ctypes.c_int32 * 3, ctypes.c_int32 * 3, i32, dbl, i32, P19],
                               ctypes.c_int),
    }
    # every entry point gets a prototype: an unprototyped call would pass pointers as C ints
    missing = [name for name in EXPORTED if name not in sig]
    if missing:
        raise ImportError(f"no ctypes prototype for {missing}")
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


lib = _load()


def _check(rc: int, handle=None):
    if rc != 0:
        raise EupError(rc, lib.eup_last_error(handle).decode(errors="replace"))


def device_count() -> int:
    return int(lib.eup_device_count())


def _ptrs(arr: np.ndarray):
    assert arr.ndim == 4 and arr.shape[0] == 19 and arr.flags["C_CONTIGUOUS"]
    return (ctypes.c_void_p * 19)(*[arr[q].ctypes.data for q in range(19)])


def _elem(arr: np.ndarray) -> int:
    if arr.dtype == np.float32:
        return 4
    if arr.dtype == np.float64:
        return 8
    raise TypeError("populations must be float32 or float64")


@dataclasses.dataclass
class Config:
    lx: int
    ly: int
    lz: int
    bc: tuple = (OUTFLOW, INFLOW, FREESLIP, FREESLIP, PERIODIC, PERIODIC)
    svisc: float = 0.01
    u0: float = 0.0
    u_inflow: float = 0.0
    u00: float = 0.0
    precision: int = FP32
    device: int = 0
    dev_scale: float = 0.0
    cd_rho0: float = 1.0
    cd_uref: float = 0.0
    cd_length: float = 0.0
    cd_span: float = 0.0
    series_capacity: int = 0

    def to_c(self) -> CConfig:
        c = CConfig()
        c.lx, c.ly, c.lz = self.lx, self.ly, self.lz
        for f in range(6):
            c.bc[f] = int(self.bc[f])
        c.svisc, c.u0, c.u_inflow, c.u00 = self.svisc, self.u0, self.u_inflow, self.u00
        c.precision, c.device, c.dev_scale = self.precision, self.device, self.dev_scale
        c.cd_rho0, c.cd_uref, c.cd_length, c.cd_span = self.cd_rho0, self.cd_uref, self.cd_length, self.cd_span
        c.series_capacity = self.series_capacity
        return c


class Solver:
    """One lattice on one GPU: the Python face of an eup_handle."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        h = ctypes.c_void_p()
        _check(lib.eup_create(ctypes.byref(cfg.to_c()), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib.eup_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        _check(rc, self._h)

    @property
    def shape(self):
        return (19, self.cfg.lz + 2, self.cfg.ly + 2, self.cfg.lx + 2)

    def set_obstacles(self, obs: np.ndarray):
        obs = np.ascontiguousarray(obs, dtype=np.int32)
        assert obs.shape == (self.cfg.lz, self.cfg.ly, self.cfg.lx)
        self._ck(lib.eup_set_obstacles(self._h, obs.ctypes.data))

    def build_obstacles(self, geom: Geometry):
        """Voxelises geom on the device into the solid mask and installs it (eup_build_obstacles)."""
        self._ck(lib.eup_build_obstacles(self._h, ctypes.byref(geom)))

    def obstacles(self) -> tuple[np.ndarray, int]:
        """The installed mask obs (n, m, l) and its number of solid voxels."""
        obs = np.empty((self.cfg.lz, self.cfg.ly, self.cfg.lx), dtype=np.int32)
        n = ctypes.c_int64(0)
        self._ck(lib.eup_get_obstacles(self._h, obs.ctypes.data, ctypes.byref(n)))
        return obs, int(n.value)

    def obstacle_count(self) -> int:
        """Solid voxels of the installed mask (nothing crosses to the host but the count)."""
        n = ctypes.c_int64(0)
        self._ck(lib.eup_get_obstacles(self._h, None, ctypes.byref(n)))
        return int(n.value)

    def write_obstacles(self, path: str):
        """The installed mask as an obstacle file obs.RRRR.TTTTTTTT.bin, listed on the device."""
        self._ck(lib.eup_write_obstacles(self._h, os.fsencode(str(path))))

    def upload(self, pops: np.ndarray, itime: int = 0):
        pops = np.ascontiguousarray(pops)
        assert pops.shape == self.shape
        self._ck(lib.eup_upload(self._h, _ptrs(pops), _elem(pops), itime))

    def upload_ptrs(self, ptrs, elem_bytes: int, itime: int = 0):
        """Upload from 19 raw host pointers (e.g. pinned torch tensors)."""
        self._ck(lib.eup_upload(self._h, (ctypes.c_void_p * 19)(*ptrs), elem_bytes, itime))

    def download(self, dtype=np.float32) -> np.ndarray:
        out = np.empty(self.shape, dtype=dtype)
        self._ck(lib.eup_download(self._h, _ptrs(out), _elem(out)))
        return out

    def download_ptrs(self, ptrs, elem_bytes: int):
        self._ck(lib.eup_download(self._h, (ctypes.c_void_p * 19)(*ptrs), elem_bytes))

    def step(self, nsteps: int = 1):
        self._ck(lib.eup_step(self._h, nsteps))

    def step_profiled(self, nsteps: int) -> np.ndarray:
        ms = np.zeros(4, dtype=np.float64)
        self._ck(lib.eup_step_profiled(self._h, nsteps, ms.ctypes.data))
        return ms

    def synchronize(self):
        self._ck(lib.eup_synchronize(self._h))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._ck(lib.eup_get_stream(self._h, ctypes.byref(s)))
        return int(s.value or 0)

    @property
    def launches(self) -> int:
        """Kernels launched so far by the time-step entry points."""
        t = ctypes.c_int64()
        self._ck(lib.eup_get_launch_count(self._h, ctypes.byref(t)))
        return int(t.value)

    @property
    def itime(self) -> int:
        t = ctypes.c_int64()
        self._ck(lib.eup_get_itime(self._h, ctypes.byref(t)))
        return int(t.value)

    def forces(self) -> np.ndarray:
        out = np.zeros(3, dtype=np.float64)
        self._ck(lib.eup_get_forces(self._h, out.ctypes.data))
        return out

    def force_series(self, first: int, count: int) -> np.ndarray:
        out = np.zeros((count, 3), dtype=np.float64)
        self._ck(lib.eup_get_force_series(self._h, first, count, out.ctypes.data))
        return out

    def cd_series(self, first: int, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.float64)
        self._ck(lib.eup_get_cd_series(self._h, first, count, out.ctypes.data))
        return out

    def monitor(self) -> np.ndarray:
        out = np.zeros(5, dtype=np.float64)
        self._ck(lib.eup_get_monitor(self._h, out.ctypes.data))
        return out

    def probes(self, ijk) -> np.ndarray:
        ijk = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        out = np.zeros((ijk.shape[0], 4), dtype=np.float64)
        self._ck(lib.eup_get_probes(self._h, ijk.shape[0], ijk.ctypes.data, out.ctypes.data))
        return out

    def init_state(self, u_in, amp, seed, itime=0):
        """Seeded equilibrium state generated on the device (same bits as upload(init_equilibrium(...)))."""
        self._ck(lib.eup_init_state(self._h, float(u_in), float(amp), int(seed), int(itime)))

    def step_boundaries(self):
        """First half of an x-slab step: bounce-back + force, halo planes (asynchronous)."""
        self._ck(lib.eup_step_boundaries(self._h))

    def step_stream(self):
        """Second half of an x-slab step: stream-collide, step counter (asynchronous)."""
        self._ck(lib.eup_step_stream(self._h))

    def step_stream_interior(self):
        """step_stream's columns 2..l-1, which need no received planes (asynchronous)."""
        self._ck(lib.eup_step_stream_interior(self._h))

    def step_stream_faces(self):
        """step_stream's columns 1 and l, after the planes are in, and the step counter."""
        self._ck(lib.eup_step_stream_faces(self._h))

    def get_x_planes(self, side, dev_ptr):
        """Pack the 5 populations leaving through x = 1 (side 0) or x = l (side 1) into device memory."""
        self._ck(lib.eup_get_x_planes(self._h, side, dev_ptr))

    def set_x_planes(self, side, dev_ptr):
        """Write received planes into the x = 0 (side 0) or x = l+1 (side 1) halo."""
        self._ck(lib.eup_set_x_planes(self._h, side, dev_ptr))

    def x_planes_view(self, side) -> int:
        """Device address of the plane message of an exchange face inside the handle's x-face
        copy (written by the stream-collide epilogue, halo rows added by step_boundaries):
        5 (m+2)(n+2) values, the five populations' m x n interior blocks and their halo rows
        (side 1: blocks then halo rows; side 0: halo rows then blocks)."""
        p = ctypes.c_void_p()
        self._ck(lib.eup_get_x_planes_view(self._h, side, ctypes.byref(p)))
        return p.value

    def set_x_planes_view(self, side, dev_ptr):
        """Write a message from the neighbour's opposite side (its x_planes_view order) into the
        x = 0 (side 0) / x = l+1 (side 1) halo."""
        self._ck(lib.eup_set_x_planes_view(self._h, side, dev_ptr))

    def save_state(self, path, elem_bytes=4):
        """Checkpoint in the reference's raw format straight from the device."""
        self._ck(lib.eup_save_state(self._h, os.fsencode(str(path)), elem_bytes))

    def restore_state(self, path, elem_bytes=4):
        """Restart from a file in the reference's raw format (sets the step counter)."""
        self._ck(lib.eup_restore_state(self._h, os.fsencode(str(path)), elem_bytes))

    def line(self, axis, c1, c2) -> np.ndarray:
        """prof_i/prof_j/prof_k line (axis 0/1/2) at the fixed coordinates c1, c2: rows (u, w, v, den)."""
        n = (self.cfg.lx, self.cfg.ly, self.cfg.lz)[axis]
        out = np.zeros((n, 4), dtype=np.float64)
        self._ck(lib.eup_get_line(self._h, axis, c1, c2, out.ctypes.data))
        return out

    def plane_means(self, axis=2) -> np.ndarray:
        """varm-style means (u, w, v, den) of every plane normal to axis."""
        n = (self.cfg.lx, self.cfg.ly, self.cfg.lz)[axis]
        out = np.zeros((n, 4), dtype=np.float64)
        self._ck(lib.eup_get_plane_means(self._h, axis, out.ctypes.data))
        return out

    def cv_drag(self, box) -> np.ndarray:
        """Control-volume drag (fluxX, fluxY) of box (xstart, xstop, ystart, ystop, zstart, zstop)."""
        b = np.ascontiguousarray(np.asarray(box, dtype=np.int32))
        out = np.zeros(2, dtype=np.float64)
        self._ck(lib.eup_get_cv_drag(self._h, b.ctypes.data, out.ctypes.data))
        return out

    def region_sums(self, region) -> np.ndarray:
        """FP64 {count, sum rho, sum ux, sum uy, sum uz, sum u^2} over the fluid nodes where
        region (shape (n, m, l), truthy = included) is set."""
        r = np.ascontiguousarray(np.asarray(region, dtype=bool).astype(np.uint8))
        assert r.shape == (self.cfg.lz, self.cfg.ly, self.cfg.lx)
        out = np.zeros(6, dtype=np.float64)
        self._ck(lib.eup_get_region_sums(self._h, r.ctypes.data, out.ctypes.data))
        return out

    def links(self) -> np.ndarray:
        out = np.zeros((self.cfg.lz, self.cfg.ly, self.cfg.lx), dtype=np.uint32)
        self._ck(lib.eup_get_links(self._h, out.ctypes.data))
        return out

    def set_solid_fraction(self, ns):
        """Partial-bounce-back solid fraction n_s(1:l,1:m,1:n) in [0,1] (shape (n, m, l)); None switches it off."""
        if ns is None:
            self._ck(lib.eup_set_solid_fraction(self._h, None))
            return
        ns = np.ascontiguousarray(ns, dtype=np.float64)
        assert ns.shape == (self.cfg.lz, self.cfg.ly, self.cfg.lx)
        self._keep_ns = ns
        self._ck(lib.eup_set_solid_fraction(self._h, ns.ctypes.data))

    def adjoint(self, nsteps: int, avg_steps: int, checkpoints: int = 0):
        """Runs nsteps forward and the discrete adjoint back: returns (objective = mean C_d over the
        last avg_steps steps, dJ/dn_s of shape (n, m, l), stats dict)."""
        cfg = AdjointConfig(nsteps, avg_steps, checkpoints, 0)
        obj = ctypes.c_double()
        grad = np.zeros((self.cfg.lz, self.cfg.ly, self.cfg.lx), dtype=np.float64)
        st = np.zeros(8, dtype=np.float64)
        self._ck(lib.eup_adjoint_run(self._h, ctypes.byref(cfg), ctypes.byref(obj), grad.ctypes.data, st.ctypes.data))
        keys = ["forward_ms", "reverse_ms", "recomputed_steps", "checkpoints", "repetitions", "state_bytes",
                "nsteps", "avg_steps"]
        return obj.value, grad, dict(zip(keys, st.tolist()))

    def boundary_solid(self) -> np.ndarray:
        cnt = ctypes.c_int64()
        self._ck(lib.eup_get_boundary_solid(self._h, None, 0, ctypes.byref(cnt)))
        out = np.zeros(max(cnt.value, 1), dtype=np.int64)
        self._ck(lib.eup_get_boundary_solid(self._h, out.ctypes.data, cnt.value, ctypes.byref(cnt)))
        return out[:cnt.value]


# ---- host utilities ------------------------------------------------------------

def adjoint_plan(nsteps: int, checkpoints: int = 0) -> dict:
    """The checkpoint schedule of Solver.adjoint for nsteps steps and `checkpoints` stored states
    (0: 64), computed on the host: forward steps in all, recomputed in the reverse sweep, r."""
    fwd, rec, rep = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    _check(lib.eup_adjoint_plan(int(nsteps), int(checkpoints), ctypes.byref(fwd), ctypes.byref(rec), ctypes.byref(rep)))
    return {"forward_steps": fwd.value, "recomputed_steps": rec.value, "repetitions": rep.value}


def init_equilibrium(l, m, n, u_in, amp, seed, dtype=np.float32) -> np.ndarray:
    """Synthetic initial state: equilibrium at rho=1, u = inlet + seeded perturbation, halos included."""
    out = np.empty((19, n + 2, m + 2, l + 2), dtype=dtype)
    _check(lib.eup_init_equilibrium(l, m, n, float(u_in), float(amp), int(seed), _elem(out), _ptrs(out)))
    return out


def init_reference(opt, l, m, n, glob=None, start=(0, 0, 0), periodic=False, u0=0.0, dtype=np.float32) -> np.ndarray:
    """The reference's initial state init(opt) (CODE/SRC/init.F90, options 0..3) for a block
    l x m x n at start of a glob = (lx, ly, lz) lattice, halos included."""
    out = np.empty((19, n + 2, m + 2, l + 2), dtype=dtype)
    g = (ctypes.c_int32 * 3)(*(glob if glob is not None else (l, m, n)))
    _check(lib.eup_init_reference(int(opt), l, m, n, g, (ctypes.c_int32 * 3)(*start), int(bool(periodic)),
                                  float(u0), _elem(out), _ptrs(out)))
    return out


def read_obs_file(path, l, m, n):
    obs = np.zeros((n, m, l), dtype=np.int32)
    cnt = ctypes.c_int64()
    _check(lib.eup_read_obs_file(os.fsencode(path), l, m, n, obs.ctypes.data, ctypes.byref(cnt)))
    return obs, int(cnt.value)


def write_obs_file(path, obs: np.ndarray):
    obs = np.ascontiguousarray(obs, dtype=np.int32)
    n, m, l = obs.shape
    _check(lib.eup_write_obs_file(os.fsencode(path), l, m, n, obs.ctypes.data))


def read_raw_state(path, l, m, n, dtype=np.float32):
    out = np.empty((19, n + 2, m + 2, l + 2), dtype=dtype)
    it = ctypes.c_int64()
    _check(lib.eup_read_raw_state(os.fsencode(path), l, m, n, _elem(out), _ptrs(out), ctypes.byref(it)))
    return out, int(it.value)


def write_raw_state(path, pops: np.ndarray, itime: int):
    pops = np.ascontiguousarray(pops)
    _, n2, m2, l2 = pops.shape
    _check(lib.eup_write_raw_state(os.fsencode(path), l2 - 2, m2 - 2, n2 - 2, _elem(pops), _ptrs(pops), itime))


def geometry_reference(flag2: int, lx: int, ly: int, lz: int, cylinder_inf: bool = False,
                       test1: bool = False) -> Geometry:
    """The obstacle CODE/SRC/build.obs.F90 creates for flag1 = 2 and this flag2 (1 sphere,
    2 column, 3 half column) on the global lattice lx x ly x lz."""
    g = Geometry()
    variant = (GEOM_VARIANT_CYLINDER_INF if cylinder_inf else 0) | (GEOM_VARIANT_TEST1 if test1 else 0)
    _check(lib.eup_geometry_reference(int(flag2), int(lx), int(ly), int(lz), variant, ctypes.byref(g)))
    return g


def voxelise(geom: Geometry, l: int, m: int, n: int) -> np.ndarray:
    """The host voxeliser: obs (n, m, l) of geom, identical to the device's mask."""
    obs = np.empty((n, m, l), dtype=np.int32)
    _check(lib.eup_voxelise(ctypes.byref(geom), int(l), int(m), int(n), obs.ctypes.data))
    return obs


def geometry_cylinder_z(l, m, n, xc, yc, r) -> np.ndarray:
    obs = np.zeros((n, m, l), dtype=np.int32)
    _check(lib.eup_geometry_cylinder_z(l, m, n, float(xc), float(yc), float(r), obs.ctypes.data))
    return obs


def geometry_reticular_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, seed) -> np.ndarray:
    obs = np.zeros((n, m, l), dtype=np.int32)
    _check(lib.eup_geometry_reticular_shell(l, m, n, float(x0), float(length), float(yc), float(zc),
                                            float(outer_d), float(strut_d), float(pitch), int(seed),
                                            obs.ctypes.data))
    return obs


def geometry_ridged_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, ridge_h, ridge_t, cap_t, pore_d,
                          smooth_w, seed, with_derivative=False):
    """Ridged reticular shell with a porous cap as a solid fraction (n, m, l); with
    with_derivative also d ns / d ridge_h."""
    ns = np.zeros((n, m, l), dtype=np.float64)
    d = np.zeros_like(ns) if with_derivative else None
    _check(lib.eup_geometry_ridged_shell(l, m, n, float(x0), float(length), float(yc), float(zc), float(outer_d),
                                         float(strut_d), float(pitch), float(ridge_h), float(ridge_t), float(cap_t),
                                         float(pore_d), float(smooth_w), int(seed), ns.ctypes.data,
                                         d.ctypes.data if d is not None else None))
    return (ns, d) if with_derivative else ns

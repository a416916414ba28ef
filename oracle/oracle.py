"""ctypes harness for the CPU ORACLE (test infrastructure only).

The oracle (oracle/orc.c, oracle/orc_impl.h) is a plain-C restatement of the
reference's serial D3Q19 BGK step; it is the checker for the CUDA path and the
CPU baseline leg of the benchmark.  Nothing in the product package imports
this module.  PARITY STATUS: parity unpinned (the reference has no tests or
golden vectors and cannot be compiled here).

Arrays follow the reference layout: populations as one numpy array of shape
(19, n+2, m+2, l+2) -- C order with the last axis fastest, i.e. the Fortran
arrays a01..a19(0:l+1, 0:m+1, 0:n+1) of CODE/SRC/alloca.F90:94-132 stacked.
`obs` has shape (n, m, l), 1 = solid.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")

FRONT, REAR, RIGHT, LEFT, UP, DOWN = range(6)
PERIODIC, NOSLIP, LID, FREESLIP, INFLOW, OUTFLOW = range(6)


class Params(ctypes.Structure):
    _fields_ = [
        ("l", ctypes.c_int32), ("m", ctypes.c_int32), ("n", ctypes.c_int32),
        ("bc", ctypes.c_int32 * 6),
        ("svisc", ctypes.c_double), ("u0", ctypes.c_double),
        ("u_inflow", ctypes.c_double), ("u00", ctypes.c_double),
    ]


def build() -> str:
    """Compile the oracle library in place (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        PP = ctypes.POINTER(ctypes.c_void_p)
        for pfx in ("f", "d"):
            getattr(L, f"orc_{pfx}_run").argtypes = [ctypes.POINTER(Params), PP, PP, ctypes.c_void_p, ctypes.c_int32]
            getattr(L, f"orc_{pfx}_run").restype = ctypes.c_int
            for nm in ("bcond_obs",):
                getattr(L, f"orc_{pfx}_{nm}").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_bcond_bc").argtypes = [ctypes.POINTER(Params), PP]
            getattr(L, f"orc_{pfx}_movef").argtypes = [ctypes.POINTER(Params), PP, PP]
            getattr(L, f"orc_{pfx}_col").argtypes = [ctypes.POINTER(Params), PP, PP]
            getattr(L, f"orc_{pfx}_init_perturbed").argtypes = [
                ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                ctypes.c_uint64, PP]
            I3 = ctypes.c_int32 * 3
            getattr(L, f"orc_{pfx}_init_reference").argtypes = [
                ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, I3, I3, ctypes.c_int32,
                ctypes.c_double, PP]
            getattr(L, f"orc_{pfx}_init_reference").restype = ctypes.c_int
            getattr(L, f"orc_{pfx}_mem_force").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_void_p, ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_monitor").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_void_p, ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_macro").argtypes = [ctypes.POINTER(Params), PP] + [ctypes.c_void_p] * 4
            getattr(L, f"orc_{pfx}_constants").argtypes = [ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_line").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_int32, ctypes.c_int32,
                                                      ctypes.c_int32, ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_plane_means").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_int32,
                                                             ctypes.c_void_p]
            getattr(L, f"orc_{pfx}_cv_drag").argtypes = [ctypes.POINTER(Params), PP, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_links.argtypes = [ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p]
        L.orc_boundary_solid.argtypes = [ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p]
        L.orc_boundary_solid.restype = ctypes.c_int64
        dbl = ctypes.c_double
        L.orc_voxelise_shell.argtypes = [ctypes.c_int32] * 3 + [dbl] * 7 + [ctypes.c_uint64, ctypes.c_void_p]
        L.orc_voxelise_shell.restype = ctypes.c_int64
        L.orc_voxelise_cylinder_z.argtypes = [ctypes.c_int32] * 3 + [dbl] * 3 + [ctypes.c_void_p]
        L.orc_voxelise_cylinder_z.restype = ctypes.c_int64
        L.orc_splitmix64.argtypes = [ctypes.c_uint64]
        L.orc_splitmix64.restype = ctypes.c_uint64
        L.orc_nthreads.restype = ctypes.c_int32
        _lib = L
    return _lib


def params(l, m, n, bc, svisc, u0=0.0, u_inflow=0.0, u00=0.0) -> Params:
    p = Params()
    p.l, p.m, p.n = l, m, n
    for f in range(6):
        p.bc[f] = int(bc[f])
    p.svisc, p.u0, p.u_inflow, p.u00 = float(svisc), float(u0), float(u_inflow), float(u00)
    return p


def _pfx(arr: np.ndarray) -> str:
    if arr.dtype == np.float32:
        return "f"
    if arr.dtype == np.float64:
        return "d"
    raise TypeError(f"populations must be float32 or float64, got {arr.dtype}")


def _ptrs(arr: np.ndarray):
    assert arr.flags["C_CONTIGUOUS"] and arr.shape[0] == 19
    return (ctypes.c_void_p * 19)(*[arr[q].ctypes.data for q in range(19)])


def _obs_ptr(obs):
    if obs is None:
        return None
    assert obs.dtype == np.int32 and obs.flags["C_CONTIGUOUS"]
    return obs.ctypes.data


def new_state(l, m, n, dtype=np.float32) -> np.ndarray:
    # CODE/SRC/alloca.F90:134-172 fills fresh arrays with huge(); every value read
    # by the step is overwritten by init or restore before use.
    return np.full((19, n + 2, m + 2, l + 2), 3.0e38 if dtype == np.float32 else 1.0e300, dtype=dtype)


def init_perturbed(l, m, n, u_in, amp, seed, dtype=np.float32) -> np.ndarray:
    a = new_state(l, m, n, dtype)
    getattr(lib(), f"orc_{_pfx(a)}_init_perturbed")(l, m, n, u_in, amp, seed, _ptrs(a))
    return a


def init_reference(opt, l, m, n, glob=None, start=(0, 0, 0), periodic=False, u0=0.0, dtype=np.float32):
    """init(opt) of CODE/SRC/init.F90 (options 0..3) on a block of a glob lattice."""
    a = new_state(l, m, n, dtype)
    g = (ctypes.c_int32 * 3)(*(glob if glob is not None else (l, m, n)))
    st = (ctypes.c_int32 * 3)(*start)
    rc = getattr(lib(), f"orc_{_pfx(a)}_init_reference")(opt, l, m, n, g, st, int(bool(periodic)), float(u0),
                                                           _ptrs(a))
    if rc != 0:
        raise ValueError(f"init option {opt} not restated")
    return a


def run(p: Params, a: np.ndarray, obs: np.ndarray | None, nsteps: int, b: np.ndarray | None = None) -> np.ndarray:
    """Advance `a` in place by nsteps reference time steps; returns the scratch b."""
    if b is None:
        b = np.zeros_like(a)
    rc = getattr(lib(), f"orc_{_pfx(a)}_run")(ctypes.byref(p), _ptrs(a), _ptrs(b), _obs_ptr(obs), nsteps)
    assert rc == 0
    return b


def bcond_obs(p, a, obs):
    getattr(lib(), f"orc_{_pfx(a)}_bcond_obs")(ctypes.byref(p), _ptrs(a), _obs_ptr(obs))


def bcond_bc(p, a):
    getattr(lib(), f"orc_{_pfx(a)}_bcond_bc")(ctypes.byref(p), _ptrs(a))


def movef(p, a, b):
    getattr(lib(), f"orc_{_pfx(a)}_movef")(ctypes.byref(p), _ptrs(a), _ptrs(b))


def col(p, a, b):
    getattr(lib(), f"orc_{_pfx(a)}_col")(ctypes.byref(p), _ptrs(a), _ptrs(b))


def constants(p, dtype=np.float32):
    o = np.zeros(1, dtype=dtype)
    f = np.zeros(1, dtype=dtype)
    getattr(lib(), f"orc_{'f' if dtype == np.float32 else 'd'}_constants")(ctypes.byref(p), o.ctypes.data, f.ctypes.data)
    return o[0], f[0]


def mem_force(p, a, obs) -> np.ndarray:
    out = np.zeros(3, dtype=np.float64)
    getattr(lib(), f"orc_{_pfx(a)}_mem_force")(ctypes.byref(p), _ptrs(a), _obs_ptr(obs), out.ctypes.data)
    return out


def monitor(p, a, obs) -> np.ndarray:
    out = np.zeros(5, dtype=np.float64)
    getattr(lib(), f"orc_{_pfx(a)}_monitor")(ctypes.byref(p), _ptrs(a), _obs_ptr(obs), out.ctypes.data)
    return out


def macro(p, a):
    shp = (p.n, p.m, p.l)
    rho, ux, uy, uz = (np.zeros(shp, dtype=np.float64) for _ in range(4))
    getattr(lib(), f"orc_{_pfx(a)}_macro")(ctypes.byref(p), _ptrs(a), rho.ctypes.data, ux.ctypes.data,
                                           uy.ctypes.data, uz.ctypes.data)
    return rho, ux, uy, uz


def line(p, a, axis, c1, c2) -> np.ndarray:
    """prof_i/prof_j/prof_k line (axis 0/1/2): rows (u, w, v, den) per node, computed in the state's type."""
    n = (p.l, p.m, p.n)[axis]
    out = np.zeros((n, 4), dtype=np.float64)
    getattr(lib(), f"orc_{_pfx(a)}_line")(ctypes.byref(p), _ptrs(a), axis, c1, c2, out.ctypes.data)
    return out


def plane_means(p, a, axis) -> np.ndarray:
    """varm-style plane means (u, w, v, den) of every plane normal to axis, FP64 accumulation."""
    n = (p.l, p.m, p.n)[axis]
    out = np.zeros((n, 4), dtype=np.float64)
    getattr(lib(), f"orc_{_pfx(a)}_plane_means")(ctypes.byref(p), _ptrs(a), axis, out.ctypes.data)
    return out


def cv_drag(p, a, box) -> np.ndarray:
    """Control-volume drag (fluxX, fluxY) of the box (xstart, xstop, ystart, ystop, zstart, zstop)."""
    b = np.ascontiguousarray(np.asarray(box, dtype=np.int32))
    out = np.zeros(2, dtype=np.float64)
    getattr(lib(), f"orc_{_pfx(a)}_cv_drag")(ctypes.byref(p), _ptrs(a), b.ctypes.data, out.ctypes.data)
    return out


def links(p, obs) -> np.ndarray:
    out = np.zeros((p.n, p.m, p.l), dtype=np.uint32)
    lib().orc_links(ctypes.byref(p), _obs_ptr(obs), out.ctypes.data)
    return out


def boundary_solid(p, obs) -> np.ndarray:
    cnt = lib().orc_boundary_solid(ctypes.byref(p), _obs_ptr(obs), None)
    out = np.zeros(max(cnt, 1), dtype=np.int64)
    lib().orc_boundary_solid(ctypes.byref(p), _obs_ptr(obs), out.ctypes.data)
    return out[:cnt]


def voxelise_shell(l, m, n, x0, length, yc, zc, outer_d, strut_d, pitch, seed) -> np.ndarray:
    """The reticular shell of the benchmark workloads as obs (n, m, l) (oracle/orc_geom.c)."""
    obs = np.empty((n, m, l), dtype=np.int32)
    lib().orc_voxelise_shell(l, m, n, float(x0), float(length), float(yc), float(zc), float(outer_d),
                             float(strut_d), float(pitch), int(seed), obs.ctypes.data)
    return obs


def voxelise_cylinder_z(l, m, n, xc, yc, r) -> np.ndarray:
    """Solid circular cylinder along z, (i - xc)^2 + (j - yc)^2 <= r^2, as obs (n, m, l)."""
    obs = np.empty((n, m, l), dtype=np.int32)
    lib().orc_voxelise_cylinder_z(l, m, n, float(xc), float(yc), float(r), obs.ctypes.data)
    return obs


def nthreads() -> int:
    return int(lib().orc_nthreads())


def created_obstacle(flag2, lx, ly, lz, l, m, n, mpicoords=(0, 0, 0), cylinder_inf=False, test1=False):
    """Obstacle of CODE/SRC/build.obs.F90 for flag1 = 2 on the local block (l, m, n) at
    process coordinates mpicoords of a global lx x ly x lz lattice, restated line by line:
    flag2 = 1 sphere (:207-268), 2 column (:271-367), 3 half column (:370-441), with d2
    formed in integers and compared in the reference's single-precision reals.  Returns
    (obs (n, m, l) int32, nobs) where nobs is the reference's counter after the loop: it
    starts at -100 (:68), so it is the number of solid voxels minus 100."""
    f32 = np.float32
    offx, offy, offz = mpicoords[0] * l, mpicoords[1] * m, mpicoords[2] * n
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    if flag2 == 1:
        icoord, jcoord, kcoord = lx // 4, ly // 2, lz // 2
        radius = min(ly // 4, lz // 4) if test1 else 20
        R = f32(radius * 1.0)
        R2a, R2b = f32((R - f32(2)) * (R - f32(2))), f32((R + f32(2)) * (R + f32(2)))
        d2i = (icoord - (i + offx)) ** 2 + (jcoord - (j + offy)) ** 2 + (kcoord - (k + offz)) ** 2
        d2 = d2i.astype(f32)
        obs = (d2 > R2a) & (d2 < R2b)
    elif flag2 in (2, 3):
        if flag2 == 2 and cylinder_inf:
            radius, icoord, jcoord, kcoord, size_z = 100, lx // 4, ly // 2, 0, lz + 1
        elif flag2 == 2:
            radius, icoord, jcoord, kcoord, size_z = min(20, lx // 8), lx // 4, ly // 2, 0, lz
        else:
            radius, icoord, jcoord, kcoord, size_z = min(20, lz // 8), lx // 4, ly // 2, 0, 60
        start_z = kcoord - mpicoords[2] * n
        stop_z = start_z + size_z
        R = f32(radius * 1.0)
        R2a, R2b = f32(0), f32((R + f32(2)) * (R + f32(2)))
        d2 = ((icoord - (i + offx)) ** 2 + (jcoord - (j + offy)) ** 2).astype(f32)
        obs = (k >= start_z) & (k < stop_z) & (d2 >= R2a) & (d2 < R2b)
    else:
        raise ValueError("flag2 must be 1, 2 or 3")
    obs = obs.astype(np.int32)
    return obs, int(obs.sum()) - 100


def obstacle_file_bytes(obs, count=None) -> bytes:
    """The obstacle dump of CODE/SRC/build.obs.F90:506-541 as gfortran writes it: a record
    holding the count, then one (i, j, k) record per solid voxel, i fastest.  count defaults
    to the number of solid voxels."""
    kk, jj, ii = np.nonzero(np.asarray(obs) == 1)  # C order over (n, m, l): i fastest
    nobs = len(ii) if count is None else count
    rec = np.empty((len(ii), 5), dtype=np.int32)
    rec[:, 0] = rec[:, 4] = 12
    rec[:, 1], rec[:, 2], rec[:, 3] = ii + 1, jj + 1, kk + 1
    head = np.array([4, nobs, 4], dtype=np.int32)
    return head.tobytes() + rec.tobytes()

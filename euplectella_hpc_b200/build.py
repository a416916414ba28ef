"""Builds the sm_100a shared library `_lib/libeup.so` in place with nvcc.

Every CUDA translation unit is compiled for `sm_100a` only, with
`--fmad=false` (host code: `-ffp-contract=off`) so that each floating-point
operation rounds on its own, in source order (the FP32/FP64 step then matches
an IEEE build of the reference's Fortran bit for bit, and the host and device
voxelisers agree).  The CUDA runtime is linked statically, so the library
loads on machines without a GPU driver (entry points then return
EUP_ERR_NO_DEVICE).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libeup.so")
DRIVER = os.path.join(LIB_DIR, "eup_bgk3d")

SOURCES = ["abi.cu", "k_bc.cu", "k_step.cu", "k_setup.cu", "k_adjoint.cu", "host.cpp", "noalloc.cu"]
HEADERS = ["lbm_common.cuh", "internal.h", "geometry.h", "init_eq.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-fopenmp,-Wall,-ffp-contract=off",
          "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    nv = nvcc()
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "eup.h")]
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([nv, *ARCH, *COMMON, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)

    with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        run([nv, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fopenmp", "-o", LIB, *objs, "-lgomp"])
    # the reference program's driver over the C ABI
    drv_src = os.path.join(CSRC, "driver", "eup_bgk3d.cpp")
    if force or _stale(DRIVER, [drv_src, LIB, os.path.join(ROOT, "include", "eup.h")]):
        run([shutil.which("g++") or "g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), drv_src,
             "-L", LIB_DIR, "-leup", "-Wl,-rpath,$ORIGIN", "-o", DRIVER])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))

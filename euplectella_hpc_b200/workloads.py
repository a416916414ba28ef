"""Synthetic workloads: lattice, geometry, boundary flags and physics of the
named configurations.  There are no shipped geometry files for these sizes
(the reference's production obstacles are unshipped ~1 GB .dat files), so each
geometry is voxelised from a seed-parameterised analytic description and the
initial state is a seeded equilibrium injected the way the reference restarts
from restore.*.bin.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import (FP16_DEV, FREESLIP, FP32, INFLOW, OUTFLOW, PERIODIC, Config, Geometry, geometry_ridged_shell,
               init_equilibrium, voxelise)

U_IN = 0.05          # inlet velocity of every configuration
PERTURBATION = 1e-4  # amplitude of the seeded initial velocity perturbation


def svisc_for(re: float, u: float, d: float) -> float:
    """Kinematic viscosity for Reynolds number re = u d / nu."""
    return u * d / re


@dataclasses.dataclass
class Workload:
    name: str
    cfg: Config
    obs: np.ndarray
    steps: int
    seed: int
    probes: list = dataclasses.field(default_factory=list)
    cavity: np.ndarray | None = None  # boolean mask (n, m, l) of the body cavity
    geometry: Geometry | None = None  # the body as a voxel shape (Solver.build_obstacles builds obs on the device)

    def initial_state(self, dtype=np.float32) -> np.ndarray:
        c = self.cfg
        return init_equilibrium(c.lx, c.ly, c.lz, U_IN, PERTURBATION, self.seed, dtype)

    @property
    def nodes(self) -> int:
        return self.cfg.lx * self.cfg.ly * self.cfg.lz


def cylinder_channel(lx=256, ly=128, lz=64, d=20.0, xc=64.0, yc=64.0, re=100.0, steps=2000, seed=1234,
                     precision=FP32) -> Workload:
    """Channel with a solid circular cylinder, axis along z: inlet u=0.05 at x=0,
    zero-gradient (equilibrium) outlet, free-slip y, periodic z (256x128x64, D=20, Re=100)."""
    nu = svisc_for(re, U_IN, d)
    cfg = Config(lx, ly, lz, bc=(OUTFLOW, INFLOW, FREESLIP, FREESLIP, PERIODIC, PERIODIC), svisc=nu,
                 u_inflow=U_IN, precision=precision, cd_rho0=1.0, cd_uref=U_IN, cd_length=d, cd_span=float(lz))
    geom = Geometry.cylinder_z(xc, yc, 0.5 * d)
    obs = voxelise(geom, lx, ly, lz)
    probes = [(int(xc + 2 * d), int(yc), lz // 2), (int(xc + 4 * d), int(yc + d // 2), lz // 2)]
    return Workload("cylinder_256x128x64_re100", cfg, obs, steps, seed, probes, geometry=geom)


def reticular_shell_channel(lx=768, ly=384, lz=384, outer_d=96.0, length=256.0, strut_d=4.0, pitch=16.0,
                            re=2000.0, steps=20000, seed=2024, precision=FP32, host_mask=True) -> Workload:
    """Channel 768x384x384 with a reticular cylindrical shell (outer D 96, length 256,
    axis x, struts d=4 at pitch 16 plus diagonals in alternate cells), inlet 0.05,
    free-slip y and z (the reference's FREESLIP preset, CODE/SRC/build.bcond.F90:286-315),
    Re 2000 on the shell diameter.  host_mask=False leaves obs None (build it on the device
    from `geometry`)."""
    nu = svisc_for(re, U_IN, outer_d)
    x0 = lx / 4.0
    yc = zc = (ly + 1) / 2.0
    area = math.pi * outer_d * outer_d / 4.0  # frontal disc
    cfg = Config(lx, ly, lz, bc=(OUTFLOW, INFLOW, FREESLIP, FREESLIP, FREESLIP, FREESLIP), svisc=nu,
                 u_inflow=U_IN, precision=precision, cd_rho0=1.0, cd_uref=U_IN, cd_length=outer_d,
                 cd_span=area / outer_d)
    geom = Geometry.reticular_shell(x0, length, yc, zc, outer_d, strut_d, pitch, seed)
    obs = voxelise(geom, lx, ly, lz) if host_mask else None
    yi, zi = int(round(yc)), int(round(zc))
    probes = [(int(x0 - 32), yi, zi), (int(x0 + length / 2), yi, zi), (int(x0 + length + 64), yi, zi)]
    # cavity: inside the strut centreline radius minus a strut radius, within the shell's x span
    k, j, i = np.meshgrid(np.arange(1, lz + 1), np.arange(1, ly + 1), np.arange(1, lx + 1), indexing="ij",
                          sparse=True)
    rin = 0.5 * outer_d - strut_d
    cavity = ((j - yc) ** 2 + (k - zc) ** 2 < rin * rin) & (i >= x0) & (i <= x0 + length)
    return Workload("reticular_shell_768x384x384_re2000", cfg, obs, steps, seed, probes, cavity, geom)


def _gauss(seed: int, n: int) -> np.ndarray:
    """Seeded standard normals: Box-Muller on splitmix64(seed + 2t), splitmix64(seed + 2t + 1)."""
    t = np.arange(n, dtype=np.uint64)
    def mix(x):
        with np.errstate(over="ignore"):
            z = x + np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            return z ^ (z >> np.uint64(31))
    s = np.uint64(seed)
    with np.errstate(over="ignore"):
        u1 = ((mix(s + np.uint64(2) * t) >> np.uint64(11)).astype(np.float64) + 0.5) / 9007199254740992.0
        u2 = ((mix(s + np.uint64(2) * t + np.uint64(1)) >> np.uint64(11)).astype(np.float64)) / 9007199254740992.0
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def solid_fraction_cylinder(lx, ly, lz, d, xc, yc, sigma, seed, width=1.0, band=1e-3) -> np.ndarray:
    """n_s = smoothed cylinder (axis z): 0.5 (1 - tanh((r - d/2)/width)), plus seeded
    N(0, sigma) noise on the voxels of the body, i.e. where the smoothed field exceeds
    `band` (noise on every voxel would turn the whole channel into a porous medium whose
    drag swamps the cylinder's), clamped to [0, 1]; shape (lz, ly, lx)."""
    k, j, i = np.meshgrid(np.arange(1, lz + 1), np.arange(1, ly + 1), np.arange(1, lx + 1), indexing="ij")
    r = np.sqrt((i - xc) ** 2 + (j - yc) ** 2)
    ns = 0.5 * (1.0 - np.tanh((r - 0.5 * d) / width))
    noise = sigma * _gauss(seed, lx * ly * lz).reshape(lz, ly, lx)
    ns = np.where(ns > band, ns + noise, ns)
    return np.clip(ns, 0.0, 1.0)


def pbb_cylinder_channel(lx=192, ly=96, lz=96, d=24.0, re=100.0, steps=4000, avg_steps=1000, sigma=0.05,
                         seed=4242, precision=FP32) -> Workload:
    """Adjoint workload: 192x96x96 channel (inlet 0.05, outflow, free-slip y, periodic z) holding a
    partial-bounce-back solid fraction (smoothed D=24 cylinder + seeded Gaussian noise, sigma 0.05);
    Re 100; objective mean C_d over the last 1000 of 4000 steps."""
    nu = svisc_for(re, U_IN, d)
    cfg = Config(lx, ly, lz, bc=(OUTFLOW, INFLOW, FREESLIP, FREESLIP, PERIODIC, PERIODIC), svisc=nu,
                 u_inflow=U_IN, precision=precision, cd_rho0=1.0, cd_uref=U_IN, cd_length=d, cd_span=float(lz))
    wl = Workload("pbb_cylinder_192x96x96_re100", cfg, np.zeros((lz, ly, lx), np.int32), steps, seed)
    wl.ns = solid_fraction_cylinder(lx, ly, lz, d, lx / 4.0, (ly + 1) / 2.0, sigma, seed)
    wl.avg_steps = avg_steps
    return wl


@dataclasses.dataclass
class RidgedShell:
    """Geometry parameters of the ridged lattice shell, in lattice units."""
    x0: float
    length: float
    yc: float
    zc: float
    outer_d: float
    strut_d: float
    pitch: float
    ridge_h: float
    ridge_t: float
    cap_t: float
    pore_d: float
    seed: int

    def args(self, lx, ly, lz):
        return (lx, ly, lz, self.x0, self.length, self.yc, self.zc, self.outer_d, self.strut_d, self.pitch)

    def geometry(self) -> Geometry:
        return Geometry.ridged_shell(self.x0, self.length, self.yc, self.zc, self.outer_d, self.strut_d, self.pitch,
                                     self.ridge_h, self.ridge_t, self.cap_t, self.pore_d, self.seed)

    def mask(self, lx, ly, lz) -> np.ndarray:
        """The 0/1 obstacle: the field below at smooth_w = 0, thresholded at 1/2."""
        return voxelise(self.geometry(), lx, ly, lz)

    def field(self, lx, ly, lz, smooth_w, ridge_h=None):
        """Solid fraction with smoothed ridges and d n_s / d ridge_h."""
        h = self.ridge_h if ridge_h is None else ridge_h
        return geometry_ridged_shell(*self.args(lx, ly, lz), h, self.ridge_t, self.cap_t, self.pore_d, smooth_w,
                                     self.seed, with_derivative=True)


def ridged_shell_channel(lx=1024, ly=512, lz=512, scale=1.0, re=2000.0, steps=10000, seed=2025,
                         precision=FP16_DEV, host_mask=True) -> Workload:
    """Channel 1024x512x512 holding the reticular shell of the 768x384x384 case (outer D 96,
    length 256, struts d=4 at pitch 16) plus two counter-rotating 45-degree helical ridges
    (height 8, thickness 4) and a seeded porous cap (thickness 4, pores of diameter 10 on a
    20-lu grid) at its downstream end; inlet 0.05, free-slip y and z, Re 2000 on the shell
    diameter; FP16-stored deviations.  (A cap with 6-lu pores makes the BGK run diverge within
    300 steps in every precision, FP64 included: the jets through pores that small are not
    resolved at this viscosity.)  `scale` shrinks the channel and every length of the body
    together (the viscosity follows Re on the scaled diameter).  host_mask=False leaves obs None
    (build it on the device from `geometry`)."""
    lx, ly, lz = int(round(lx * scale)), int(round(ly * scale)), int(round(lz * scale))
    body = RidgedShell(x0=lx / 4.0, length=256.0 * scale, yc=(ly + 1) / 2.0, zc=(lz + 1) / 2.0, outer_d=96.0 * scale,
                       strut_d=4.0 * scale, pitch=16.0 * scale, ridge_h=8.0 * scale, ridge_t=4.0 * scale,
                       cap_t=4.0 * scale, pore_d=10.0 * scale, seed=seed)
    nu = svisc_for(re, U_IN, body.outer_d)
    area = math.pi * body.outer_d * body.outer_d / 4.0
    cfg = Config(lx, ly, lz, bc=(OUTFLOW, INFLOW, FREESLIP, FREESLIP, FREESLIP, FREESLIP), svisc=nu,
                 u_inflow=U_IN, precision=precision, cd_rho0=1.0, cd_uref=U_IN, cd_length=body.outer_d,
                 cd_span=area / body.outer_d)
    obs = body.mask(lx, ly, lz) if host_mask else None
    yi, zi = int(round(body.yc)), int(round(body.zc))
    probes = [(int(body.x0 - 32 * scale), yi, zi), (int(body.x0 + body.length / 2), yi, zi),
              (int(body.x0 + body.length + 64 * scale), yi, zi)]
    k, j, i = np.meshgrid(np.arange(1, lz + 1), np.arange(1, ly + 1), np.arange(1, lx + 1), indexing="ij",
                          sparse=True)
    rin = 0.5 * body.outer_d - body.strut_d
    cavity = ((j - body.yc) ** 2 + (k - body.zc) ** 2 < rin * rin) & (i >= body.x0) & (i <= body.x0 + body.length)
    wl = Workload(f"ridged_shell_{lx}x{ly}x{lz}_re{int(re)}", cfg, obs, steps, seed, probes, cavity,
                  body.geometry())
    wl.body = body
    return wl

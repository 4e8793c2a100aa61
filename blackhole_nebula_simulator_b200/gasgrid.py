"""Particle -> grid deposition for the renderer on the GPU (render/gasgrid.py of the reference).

Two grids, as the reference's: ``LogSphericalGrid`` (centred on the hole, logarithmic in r,
uniform in theta and phi, phi periodic) and ``CartesianBox`` (n^3 equal cells).  A particle's
fields (m, m T, m T^4, m v) go to the cells whose centres lie inside its support (q < 2) with
weights f(q) V_c normalised to 1; fewer than 8 such centres: trilinear weights in index space
over the 8 nearest centres.  Weight beyond the grid goes to ``outside``, so grid mass + outside
= sum m for every particle.  ``deposit_log_split`` sends very wide particles to a coarser grid
whose sums are interpolated back (render/gasgrid.py:741-808).

The deposition is one warp per particle on the device (FP64 sums by atomic addition: the cell
sums are the reference's to rounding, but their last bits depend on the order the warps
arrive in); the cell fields are finished on the device too.  Inputs may be NumPy arrays or
CUDA tensors; the GasGrid fields are CUDA tensors.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from functools import cached_property

import numpy as np
import torch

from . import _lib
from .config import KERNEL_IDS
from .device import ctx, dev_f64, ptr, stream

R_SUPPORT = 2.0
MIN_KERNEL_CELLS = 8
N_FIELDS = 6  # m, m T, m T^4, m vx, m vy, m vz
INNER_VIRTUAL = 64
WIDE_CELLS = 24.0
COARSEN = (2, 4, 4)  # r, theta, phi


@dataclass(frozen=True)
class LogSphericalGrid:
    """render/gasgrid.py:52-83.  Default 192 x 96 x 192 = 3.5 M cells."""

    r_min: float = 2.0
    r_max: float = 2000.0
    nr: int = 192
    nth: int = 96
    nph: int = 192

    @cached_property
    def dlnr(self) -> float:
        return float(np.log(self.r_max / self.r_min) / self.nr)

    @cached_property
    def dth(self) -> float:
        return float(np.pi / self.nth)

    @cached_property
    def dph(self) -> float:
        return float(2.0 * np.pi / self.nph)

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.nr, self.nth, self.nph)

    def r_centres(self) -> np.ndarray:
        return self.r_min * np.exp((np.arange(self.nr) + 0.5) * self.dlnr)

    def volumes(self) -> np.ndarray:
        """Cell volumes, shape (nr, nth) (independent of phi): render/gasgrid.py:125-129."""
        i = np.arange(self.nr)[:, None]
        j = np.arange(self.nth)[None, :]
        r1 = self.r_min * np.exp(i * self.dlnr)
        r2 = r1 * np.exp(self.dlnr)
        return (r2**3 - r1**3) / 3.0 * (np.cos(j * self.dth) - np.cos((j + 1) * self.dth)) * self.dph

    def tables(self) -> dict:
        """sin / cos of the theta and phi cell centres and cos th1 - cos th2 per theta row
        (render/gasgrid.py:688-692)."""
        thc = (np.arange(self.nth) + 0.5) * self.dth
        phc = (np.arange(self.nph) + 0.5) * self.dph
        dcth = np.cos(np.arange(self.nth) * self.dth) - np.cos((np.arange(self.nth) + 1) * self.dth)
        return dict(sth=np.sin(thc), cth=np.cos(thc), dcth=dcth, cph=np.cos(phc), sph=np.sin(phc))


@dataclass(frozen=True)
class CartesianBox:
    """render/gasgrid.py:86-104: a cube of side ``size`` centred on ``centre``, n^3 cells."""

    centre: tuple[float, float, float]
    size: float
    n: int = 160

    @property
    def dx(self) -> float:
        return self.size / self.n

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.n, self.n, self.n)

    @property
    def lo(self) -> np.ndarray:
        return np.asarray(self.centre, float) - 0.5 * self.size


@dataclass
class GasGrid:
    """render/gasgrid.py:107-120: fields on one grid (float32 for rendering) and the ledger."""

    grid: object
    mass: torch.Tensor  # float64, per cell
    rho: torch.Tensor  # float32
    t_mass: torch.Tensor  # float32, K, mass-weighted (0 in empty cells)
    t_em: torch.Tensor  # float32, K, (mass-weighted mean of T^4)^(1/4)
    vel: torch.Tensor  # float32, (..., 3), mass-weighted
    outside: float  # mass deposited beyond the grid
    n_trilinear: int = 0
    extra: dict = field(default_factory=dict)


def _call(name, *args):
    c = ctx()
    _lib.check(c, getattr(_lib.lib(), name)(c, *args))


def _inputs(x, h, m, t, v):
    x = dev_f64(x)
    n = len(x)
    h = dev_f64(h, (n,))
    m = dev_f64(m, (n,))
    t = dev_f64(t, (n,))
    v = dev_f64(v, (n, 3))
    return n, x, h, m, t, v


def _check_kernel(kernel):
    if kernel not in KERNEL_IDS:
        raise ValueError(f"unknown kernel {kernel!r}; choose from {sorted(KERNEL_IDS)}")
    return KERNEL_IDS[kernel]


def _log_accumulate(x, h, m, t, v, g: LogSphericalGrid, kernel: str):
    """Accumulated sums (nr, nth, nph, N_FIELDS), outside mass, trilinear count."""
    kid = _check_kernel(kernel)
    n, x, h, m, t, v = _inputs(x, h, m, t, v)
    d = x.device
    acc = torch.empty((*g.shape, N_FIELDS), dtype=torch.float64, device=d)
    tab = {k: torch.as_tensor(a, dtype=torch.float64, device=d) for k, a in g.tables().items()}
    out = (ctypes.c_double * 1)()
    ntri = (ctypes.c_int64 * 1)()
    _call("nb_deposit_log", n, ptr(x), ptr(h), ptr(m), ptr(t), ptr(v), float(g.r_min),
          float(g.dlnr), float(g.dth), float(g.dph), int(g.nr), int(g.nth), int(g.nph), kid,
          ptr(tab["sth"]), ptr(tab["cth"]), ptr(tab["dcth"]), ptr(tab["cph"]), ptr(tab["sph"]),
          ptr(acc), out, ntri, stream())  # fmt: skip
    return acc, float(out[0]), int(ntri[0])


def _finish(g, acc, vol, outside, n_tri) -> GasGrid:
    """render/gasgrid.py:293-313 on the device; vol: (nr, nth) for the log grid (one volume per
    theta row of a shell) or a scalar for a box."""
    d = acc.device
    ncell = acc.numel() // N_FIELDS
    mass = torch.empty(acc.shape[:-1], dtype=torch.float64, device=d)
    rho, t_mass, t_em = (torch.empty(acc.shape[:-1], dtype=torch.float32, device=d) for _ in range(3))
    vel = torch.empty((*acc.shape[:-1], 3), dtype=torch.float32, device=d)
    if np.ndim(vol) == 0:
        volt = torch.full((1,), float(vol), dtype=torch.float64, device=d)
        per = ncell
    else:
        volt = torch.as_tensor(np.ascontiguousarray(vol), dtype=torch.float64, device=d)
        per = acc.shape[2]  # cells of one (i, j) row share its volume
    _call("nb_grid_finish", ncell, ptr(acc), ptr(volt), int(per), ptr(mass), ptr(rho),
          ptr(t_mass), ptr(t_em), ptr(vel), stream())
    return GasGrid(g, mass, rho, t_mass, t_em, vel, float(outside), int(n_tri))


def deposit_log(x, h, m, t, v, g: LogSphericalGrid, kernel: str = "wendland_c4") -> GasGrid:
    """render/gasgrid.py:722-738: deposition onto a log-spherical grid.  x (N, 3) positions; h
    (N,) smoothing lengths; m mass(es); t (N,) temperatures [K]; v (N, 3) velocities."""
    acc, outside, n_tri = _log_accumulate(x, h, m, t, v, g, kernel)
    return _finish(g, acc, g.volumes(), outside, n_tri)


def deposit_box(x, h, m, t, v, b: CartesianBox, kernel: str = "wendland_c4") -> GasGrid:
    """render/gasgrid.py:811-825: deposition onto a Cartesian box."""
    kid = _check_kernel(kernel)
    n, x, h, m, t, v = _inputs(x, h, m, t, v)
    acc = torch.empty((*b.shape, N_FIELDS), dtype=torch.float64, device=x.device)
    lo = b.lo
    out = (ctypes.c_double * 1)()
    ntri = (ctypes.c_int64 * 1)()
    _call("nb_deposit_box", n, ptr(x), ptr(h), ptr(m), ptr(t), ptr(v), float(lo[0]), float(lo[1]),
          float(lo[2]), float(b.dx), int(b.n), kid, ptr(acc), out, ntri, stream())  # fmt: skip
    return _finish(b, acc, b.dx**3, float(out[0]), int(ntri[0]))


def coarse_log_grid(g: LogSphericalGrid, coarsen=COARSEN) -> LogSphericalGrid:
    """render/gasgrid.py:741-748."""
    cr, ct, cp = coarsen
    if g.nr % cr or g.nth % ct or g.nph % cp:
        raise ValueError(f"grid {g.shape} not divisible by {coarsen}")
    return LogSphericalGrid(r_min=g.r_min, r_max=g.r_max, nr=g.nr // cr, nth=g.nth // ct,
                            nph=g.nph // cp)  # fmt: skip


def wide_particles(x, h, g: LogSphericalGrid, wide_cells: float = WIDE_CELLS) -> torch.Tensor:
    """render/gasgrid.py:751-754: particles whose support 2h spans >= wide_cells fine angular
    cells (r dtheta)."""
    x = dev_f64(x)
    h = dev_f64(h, (len(x),))
    r = torch.linalg.norm(x, dim=1)
    return R_SUPPORT * h >= wide_cells * torch.clamp(r, min=g.r_min) * g.dth


def refine_sums(acc_c, gc: LogSphericalGrid, g: LogSphericalGrid, coarsen=COARSEN) -> torch.Tensor:
    """render/gasgrid.py:757-788 on the device: coarse sums -> fine sums (each field's density
    interpolated trilinearly in index space at the fine centres, theta and r clamped, phi
    periodic, times the fine volume, scaled to the coarse grid's mass)."""
    out = torch.empty((*g.shape, N_FIELDS), dtype=torch.float64, device=acc_c.device)
    vc = torch.as_tensor(gc.volumes(), dtype=torch.float64, device=acc_c.device)
    vf = torch.as_tensor(g.volumes(), dtype=torch.float64, device=acc_c.device)
    cr, ct, cp = coarsen
    _call("nb_refine_sums", ptr(acc_c.contiguous()), ptr(vc), int(gc.nr), int(gc.nth), int(gc.nph),
          ptr(vf), int(g.nr), int(g.nth), int(g.nph), int(cr), int(ct), int(cp), ptr(out),
          stream())  # fmt: skip
    return out


def deposit_log_split(x, h, m, t, v, g: LogSphericalGrid, kernel: str = "wendland_c4",
                      wide_cells: float = WIDE_CELLS, coarsen=COARSEN) -> GasGrid:  # fmt: skip
    """render/gasgrid.py:791-808: very wide particles on a coarser grid, interpolated back."""
    n, x, h, m, t, v = _inputs(x, h, m, t, v)
    wide = wide_particles(x, h, g, wide_cells)
    nar = ~wide
    total, outside, n_tri = _log_accumulate(x[nar], h[nar], m[nar], t[nar], v[nar], g, kernel)
    n_wide = int(wide.sum())
    if n_wide:
        gc = coarse_log_grid(g, coarsen)
        acc_c, out_c, tri_c = _log_accumulate(x[wide], h[wide], m[wide], t[wide], v[wide], gc,
                                              kernel)  # fmt: skip
        total = total + refine_sums(acc_c, gc, g, coarsen)
        outside, n_tri = outside + out_c, n_tri + tri_c
    grid = _finish(g, total, g.volumes(), outside, n_tri)
    grid.extra["n_wide"] = n_wide
    return grid

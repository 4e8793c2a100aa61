"""Seeded synthetic initial conditions for the benchmark workloads.

The reference builds its clouds from a stored glass (sim/cloud.py:36-79); the workloads here are
defined instead by seeded jittered lattices, two colliding cylinders and a Gaussian torus, so
every generator below is this project's own.  Orbits use the reference's apocentre state on a GN
(Schwarzschild-shaped) orbit (physics/orbits.py:28-61).  Units: G = c = M_bh = 1.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import units
from .config import HFACT

GUNITS = units.GasUnits()


@dataclass
class InitialConditions:
    x: np.ndarray
    v: np.ndarray
    u: np.ndarray
    mass: np.ndarray
    h: np.ndarray  # starting guess eta (m / rho)^(1/3)
    name: str = ""


def schwarzschild_el(r_peri: float, r_apo: float) -> tuple[float, float]:
    """Energy at infinity and angular momentum of the bound orbit with these turning points,
    from E^2 = (1 - 2/r)(1 + L^2/r^2) at both radii (physics/orbits.py:28-41)."""
    u_p, u_a = 1.0 / r_peri, 1.0 / r_apo
    if not (r_apo >= r_peri > 0.0 and u_p < 0.5 - u_a - u_p):
        raise ValueError(f"no bound orbit with r_peri={r_peri}, r_apo={r_apo}")
    ap, aa = 1.0 - 2.0 / r_peri, 1.0 - 2.0 / r_apo
    l2 = (ap - aa) / (aa / r_apo**2 - ap / r_peri**2)
    return float(np.sqrt(aa * (1.0 + l2 / r_apo**2))), float(np.sqrt(l2))


def apocentre_state(r_peri: float, r_apo: float):
    """(x0, v0, p0) at apocentre on +x moving in +y (physics/orbits.py:50-61)."""
    _, ell = schwarzschild_el(r_peri, r_apo)
    f = r_apo / (r_apo - 2.0)
    x0 = np.array([r_apo, 0.0, 0.0])
    v0 = np.array([0.0, ell / (f * r_apo), 0.0])
    return x0, v0, f * v0


def _jittered_lattice(rng, spacing, lo, hi, jitter=0.15):
    axes = [np.arange(lo[c] + 0.5 * spacing, hi[c], spacing) for c in range(3)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    return g + rng.uniform(-jitter, jitter, g.shape) * spacing


def cloud(n: int = 4096, radius: float = 100.0, total_mass: float = 2.3e-8,
          t_kelvin: float = 1.0e4, r_peri: float = 1500.0, r_apo: float = 3000.0,
          kernel: str = "cubic", seed: int = 1) -> InitialConditions:  # fmt: skip
    """Uniform sphere from a seeded jittered cubic lattice (the n lattice points nearest the
    centre), centred at apocentre of the (r_peri, r_apo) GN orbit, every particle moving with the
    centre's velocity, uniform u at t_kelvin (ideal gas, gamma = 5/3)."""
    rng = np.random.default_rng(seed)
    vol = 4.0 / 3.0 * math.pi * radius**3
    spacing = (vol / n) ** (1.0 / 3.0)
    box = radius + 2.0 * spacing
    pts = _jittered_lattice(rng, spacing, (-box,) * 3, (box,) * 3)
    r = np.linalg.norm(pts, axis=1)
    pts = pts[np.argsort(r, kind="stable")[:n]]
    x0, v0, _ = apocentre_state(r_peri, r_apo)
    mass = np.full(n, total_mass / n)
    rho = total_mass / vol
    return InitialConditions(
        x=pts + x0, v=np.tile(v0, (n, 1)), u=np.full(n, units.gas_u_from_temperature(t_kelvin)),
        mass=mass, h=np.full(n, HFACT[kernel] * (total_mass / n / rho) ** (1.0 / 3.0)),
        name=f"cloud{n}",
    )  # fmt: skip


def streams(n: int = 1_048_576, radius: float = 20.0, length: float = 400.0,
            r_collide: float = 1664.0, v_rel: float = 0.056, rho_cgs: float = 1.0e-10,
            t_kelvin: float = 1.0e4, gap: float | None = None, kernel: str = "cubic",
            seed: int = 3) -> InitialConditions:  # fmt: skip
    """Two opposing cylinders (radius, length) along y meeting head-on at (r_collide, 0, 0),
    each moving at v_rel/2 toward the other, filled from seeded jittered lattices (n/2 points
    nearest each axis), uniform density rho_cgs (g/cm^3) and temperature t_kelvin.

    The streams start `gap` apart (default: one lattice spacing), inside each other's kernel
    support, so the first step's signal speeds already see the collision; a gap wider than the
    support lets the first (longest) step run through the onset of the shock unresolved."""
    rng = np.random.default_rng(seed)
    half = n // 2
    vol = math.pi * radius**2 * length
    spacing = (vol / half) ** (1.0 / 3.0)
    if gap is None:
        gap = spacing
    pts = _jittered_lattice(rng, spacing, (-radius - spacing, 0.0, -radius - spacing),
                            (radius + spacing, length, radius + spacing))  # fmt: skip
    rc = np.hypot(pts[:, 0], pts[:, 2])
    pts = pts[(pts[:, 1] >= 0.0) & (pts[:, 1] < length)]
    rc = np.hypot(pts[:, 0], pts[:, 2])
    pts = pts[np.argsort(rc, kind="stable")[:half]]
    a = pts + np.array([r_collide, 0.5 * gap, 0.0])
    b = pts * np.array([1.0, -1.0, 1.0]) + np.array([r_collide, -0.5 * gap, 0.0])
    x = np.concatenate([a, b])
    v = np.zeros_like(x)
    v[:half, 1] = -0.5 * v_rel
    v[half:, 1] = 0.5 * v_rel
    rho_code = GUNITS.density_from_si(rho_cgs * 1.0e3)
    m = rho_code * vol / half
    return InitialConditions(
        x=x, v=v, u=np.full(n, units.gas_u_from_temperature(t_kelvin)), mass=np.full(n, m),
        h=np.full(n, HFACT[kernel] * (m / rho_code) ** (1.0 / 3.0)), name=f"streams{n}",
    )  # fmt: skip


def gn_circular_speed(r):
    """Speed dx/dt of a circular GN orbit of radius r: L^2 = r^2/(r-3) (Schwarzschild circular
    orbits, which GN orbits share), p_phi = L/r and v = A p = (r-2)/r p at zero radial momentum."""
    r = np.asarray(r, float)
    ell = r / np.sqrt(r - 3.0)
    return (r - 2.0) / r * ell / r


def torus(n: int = 4_194_304, r_major: float = 100.0, a_minor: float = 40.0,
          sigma: float = 15.0, total_mass: float = 0.01, t_kelvin: float = 1.0e9,
          noise: float = 0.01, kernel: str = "cubic", seed: int = 4) -> InitialConditions:  # fmt: skip
    """Torus about the z axis (major radius r_major, minor radius a_minor) with a Gaussian density
    profile exp(-s^2 / 2 sigma^2) in the minor radius s, random seeded positions, circular GN
    velocities about z plus `noise` (relative, Gaussian per component), uniform temperature."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while len(out) < n:
        k = int((n - len(out)) * 1.6) + 1024
        s = np.abs(rng.normal(0.0, sigma, k))
        th = rng.uniform(0.0, 2.0 * math.pi, k)
        phi = rng.uniform(0.0, 2.0 * math.pi, k)
        # volume element ~ s (R + s cos th): the Gaussian in s already carries no 1/s, so keep
        # with probability s/a (R + s cos th)/(R + a) (s <= a)
        keep = (s <= a_minor) & (rng.uniform(0.0, 1.0, k) < (s / a_minor) *
                                 (r_major + s * np.cos(th)) / (r_major + a_minor))  # fmt: skip
        s, th, phi = s[keep], th[keep], phi[keep]
        cyl = r_major + s * np.cos(th)
        p = np.stack([cyl * np.cos(phi), cyl * np.sin(phi), s * np.sin(th)], axis=1)
        out = np.concatenate([out, p])
    x = out[:n]
    r = np.linalg.norm(x, axis=1)
    vc = gn_circular_speed(r)
    cyl = np.hypot(x[:, 0], x[:, 1])
    v = np.stack([-x[:, 1] / cyl, x[:, 0] / cyl, np.zeros(n)], axis=1) * vc[:, None]
    v = v + noise * vc[:, None] * rng.normal(0.0, 1.0, (n, 3))
    mass = np.full(n, total_mass / n)
    vol = 2.0 * math.pi**2 * r_major * a_minor**2
    return InitialConditions(
        x=x, v=v, u=np.full(n, units.gas_u_from_temperature(t_kelvin)), mass=mass,
        h=np.full(n, HFACT[kernel] * (total_mass / n / (total_mass / vol)) ** (1.0 / 3.0)),
        name=f"torus{n}",
    )  # fmt: skip

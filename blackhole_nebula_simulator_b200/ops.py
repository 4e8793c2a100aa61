"""The reference's inner operators on the GPU, same names, arguments and results.

Each function replaces one reference function one for one (file:line in its docstring) and runs
the sm_100a kernels of libnebula_b200.so.  Inputs may be NumPy arrays or tensors; results are
float64 / int64 CUDA tensors (``.cpu().numpy()`` gives the reference's arrays).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import torch

from . import _lib
from .config import C_NORM, DEFAULT_ETA, DEFAULT_KERNEL, KERNEL_IDS, ShockCapturing
from .device import ctx, dev_f64, dev_i64, ptr, stream

GLFConvergenceError = _lib.GLFConvergenceError

FLAG_OK, FLAG_AT_H_MAX, FLAG_SEARCH_TOO_SMALL, FLAG_NO_CONVERGENCE = 0, 1, 2, 3


def _call(name, *args):
    c = ctx()
    _lib.check(c, getattr(_lib.lib(), name)(c, *args))


@dataclass
class Neighbours:
    """CSR lists (sim/neighbours.py:22-36): neighbours of i are index[offset[i]:offset[i+1]]."""

    offset: torch.Tensor
    index: torch.Tensor
    box: object = None

    def of(self, i: int) -> torch.Tensor:
        return self.index[int(self.offset[i]) : int(self.offset[i + 1])]

    @property
    def counts(self) -> torch.Tensor:
        return torch.diff(self.offset)


def find_neighbours(pos, h, box=None) -> Neighbours:
    """sim/neighbours.py:240-281 (find_neighbours_numba): symmetric lists {j : r_ij < 2 max(h_i,
    h_j)}, self included, rows sorted.  Periodic boxes are not part of the CUDA path."""
    if box is not None:
        raise NotImplementedError("periodic boxes are not part of the CUDA SPH path")
    pos = dev_f64(pos)
    h = dev_f64(h)
    n = len(pos)
    off = torch.empty(n + 1, dtype=torch.int64, device=pos.device)
    total = ctypes.c_int64(0)
    _call("nb_find_neighbours", n, ptr(pos), ptr(h), ptr(off), ctypes.byref(total), stream())
    idx = torch.empty(max(total.value, 1), dtype=torch.int64, device=pos.device)
    _call("nb_neighbours_export", ptr(off), ptr(idx), stream())
    return Neighbours(off, idx[: total.value], None)


def cell_geometry(pos, h):
    """sim/neighbours.py:250-265 (find_neighbours_numba's grid, no periodic box): (lo, inv_cell,
    ncell) as host arrays, float64 (3), float64 (3), int64 (3)."""
    import numpy as np

    pos, h = dev_f64(pos), dev_f64(h)
    lo, ic, nc = (ctypes.c_double * 3)(), (ctypes.c_double * 3)(), (ctypes.c_int64 * 3)()
    _call("nb_cell_geometry", len(pos), ptr(pos), ptr(h), lo, ic, nc, stream())
    return np.array(lo[:]), np.array(ic[:]), np.array(nc[:], dtype=np.int64)


def build_grid(pos, lo, inv_cell, ncell):
    """sim/neighbours.py:106-126 (_build_grid): (start, order) of the stable counting sort of the
    particles by cell (cx * ny + cy) * nz + cz, as int64 CUDA tensors."""
    pos = dev_f64(pos)
    n = len(pos)
    lo3 = (ctypes.c_double * 3)(*[float(v) for v in lo])
    ic3 = (ctypes.c_double * 3)(*[float(v) for v in inv_cell])
    nc3 = (ctypes.c_int64 * 3)(*[int(v) for v in ncell])
    total = int(nc3[0]) * int(nc3[1]) * int(nc3[2])
    start = torch.empty(total + 1, dtype=torch.int64, device=pos.device)
    order = torch.empty(max(n, 1), dtype=torch.int64, device=pos.device)
    _call("nb_build_cells", n, ptr(pos), lo3, ic3, nc3, ptr(start), ptr(order), stream())
    return start, order[:n]


def tighten(nb: Neighbours, pos, h, rows=None) -> Neighbours:
    """sim/neighbours.py:306-323: keep r < 2 max(h_i, h_j), lists for ``rows`` only."""
    pos = dev_f64(pos)
    h = dev_f64(h)
    n = len(pos)
    rows_t = torch.arange(n, device=pos.device) if rows is None else dev_i64(rows)
    counts = torch.zeros(n, dtype=torch.int64, device=pos.device)
    off_in, idx_in = dev_i64(nb.offset), dev_i64(nb.index)
    _call("nb_tighten", n, ptr(pos), ptr(h), ptr(off_in), ptr(idx_in), len(rows_t), ptr(rows_t),
          ptr(counts), None, None, stream())  # fmt: skip
    off = torch.zeros(n + 1, dtype=torch.int64, device=pos.device)
    torch.cumsum(counts, 0, out=off[1:])
    total = int(off[-1])
    idx = torch.empty(max(total, 1), dtype=torch.int64, device=pos.device)
    _call("nb_tighten", n, ptr(pos), ptr(h), ptr(off_in), ptr(idx_in), len(rows_t), ptr(rows_t),
          ptr(counts), ptr(off), ptr(idx), stream())  # fmt: skip
    return Neighbours(off, idx[:total], nb.box)


@dataclass
class DensityResult:
    h: torch.Tensor
    rho: torch.Tensor
    omega: torch.Tensor
    iterations: torch.Tensor
    flags: torch.Tensor
    neighbours: Neighbours


def density_numba(pos, mass, h_start, nb: Neighbours, h_search, kernel_name=DEFAULT_KERNEL,
                  eta=DEFAULT_ETA, tol=1e-4, h_max=math.inf, rows=None) -> DensityResult:  # fmt: skip
    """sim/sph.py:300-326: the density pass on given lists; results in rows order."""
    pos = dev_f64(pos)
    n = len(pos)
    kid = KERNEL_IDS[kernel_name]
    rows_t = None if rows is None else dev_i64(rows)
    m = n if rows_t is None else len(rows_t)
    d = pos.device
    h_out, rho, om = (torch.empty(m, dtype=torch.float64, device=d) for _ in range(3))
    it, fl = (torch.empty(m, dtype=torch.int64, device=d) for _ in range(2))
    mass_t, hs_t, hsr_t = dev_f64(mass, (n,)), dev_f64(h_start, (n,)), dev_f64(h_search, (n,))
    off, idx = dev_i64(nb.offset), dev_i64(nb.index)
    _call("nb_density", n, ptr(pos), ptr(mass_t), ptr(hs_t), ptr(hsr_t), ptr(off), ptr(idx), m,
          ptr(rows_t), kid, float(eta), float(tol), float(h_max), ptr(h_out), ptr(rho), ptr(om),
          ptr(it), ptr(fl), stream())  # fmt: skip
    return DensityResult(h_out, rho, om, it, fl, nb)


FLAG_SEARCH_TOO_SMALL = 2  # sim/sph.py density flags: the search radius was too small


def compute_density(pos, mass, h_guess, kernel_name=DEFAULT_KERNEL, eta=DEFAULT_ETA, tol=1e-4,
                    h_max=math.inf, skin=1.4) -> DensityResult:  # fmt: skip
    """sim/sph.py:329-387 without a list cache (each call builds its lists): lists with search
    radius 2 min(h_guess, h_max) x skin; particles whose h outgrows the search are redone with
    rebuilt lists and their search doubled, up to 12 rounds (RuntimeError beyond)."""
    pos = dev_f64(pos)
    n = len(pos)
    h_guess = dev_f64(h_guess, (n,)).clone()
    h_search = torch.clamp(h_guess, max=h_max) * skin
    for _ in range(12):
        nb = find_neighbours(pos, h_search)
        res = density_numba(pos, mass, h_guess, nb, h_search, kernel_name, eta, tol, h_max)
        grow = res.flags == FLAG_SEARCH_TOO_SMALL
        if not bool(torch.any(grow)):
            return res
        h_search = h_search.clone()
        h_search[grow] = h_search[grow] * 2.0
        h_guess = res.h.clone()
    raise RuntimeError("smoothing lengths kept outgrowing the neighbour search")


@dataclass
class ForceResult:
    acc: torch.Tensor
    dudt: torch.Tensor
    vsig_max: torch.Tensor
    dudt_visc: torch.Tensor = None
    dudt_cond: torch.Tensor = None


def forces_numba(pos, vel, mass, h, rho, omega, pressure, nb: Neighbours,
                 kernel_name=DEFAULT_KERNEL, u=None, c_s=None, alpha=None,
                 shock: ShockCapturing = ShockCapturing(), rows=None, grad_v=None) -> ForceResult:  # fmt: skip
    """sim/sph.py:655-690: with ``shock.reconstruction`` the viscosity uses the reconstructed
    velocity jump (sim/sph.py:568-609) and needs ``grad_v`` (N, 3, 3) of all particles
    (``velocity_gradients_numba``); ValueError without it, as the reference."""
    use_visc = alpha is not None and c_s is not None
    use_recon = use_visc and shock.reconstruction
    pos = dev_f64(pos)
    n = len(pos)
    rows_t = None if rows is None else dev_i64(rows)
    m = n if rows_t is None else len(rows_t)
    d = pos.device
    acc = torch.empty((m, 3), dtype=torch.float64, device=d)
    dudt, vsig, vh, ch = (torch.empty(m, dtype=torch.float64, device=d) for _ in range(4))
    opt = lambda a: None if a is None else dev_f64(a, (n,))  # noqa: E731
    off, idx = dev_i64(nb.offset), dev_i64(nb.index)
    args = [dev_f64(vel), dev_f64(mass, (n,)), dev_f64(h), dev_f64(rho), dev_f64(omega),
            dev_f64(pressure), opt(u if use_visc else None), opt(c_s if use_visc else None),
            opt(alpha if use_visc else None)]  # fmt: skip
    if use_recon:
        if grad_v is None or tuple(grad_v.shape) != (n, 3, 3):
            raise ValueError("velocity reconstruction needs grad_v of shape (N, 3, 3)")
        gv = dev_f64(grad_v, (n, 3, 3))
        _call("nb_forces_recon", n, ptr(pos), *[ptr(a) for a in args], ptr(gv), ptr(off),
              ptr(idx), m, ptr(rows_t), KERNEL_IDS[kernel_name], float(shock.beta),
              float(shock.alpha_u), int(shock.conductivity_signal), int(bool(shock.closeness)),
              float(shock.eta_crit), float(shock.eta_fold), int(shock.recon_gate), ptr(acc),
              ptr(dudt), ptr(vsig), ptr(vh), ptr(ch), stream())  # fmt: skip
    else:
        _call("nb_forces", n, ptr(pos), *[ptr(a) for a in args], ptr(off), ptr(idx), m,
              ptr(rows_t), KERNEL_IDS[kernel_name], float(shock.beta), float(shock.alpha_u),
              int(shock.conductivity_signal), ptr(acc), ptr(dudt), ptr(vsig), ptr(vh), ptr(ch),
              stream())  # fmt: skip
    if not use_visc:
        vh.zero_()
        ch.zero_()
    return ForceResult(acc, dudt, vsig, vh, ch)


@dataclass
class Gradients:
    """sim/sph.py:708-712."""

    div_v: torch.Tensor
    curl_v: torch.Tensor  # magnitude |curl v|
    ddivv_dt: torch.Tensor


def gradients_numba(pos, vel, acc, mass, h, nb: Neighbours, kernel_name=DEFAULT_KERNEL,
                    rows=None) -> Gradients:  # fmt: skip
    """sim/sph.py:883-902: corrected div v, |curl v| and d(div v)/dt (Cullen & Dehnen 2010
    App. B3) of ``rows`` (in that order; default all) from velocities and accelerations."""
    pos = dev_f64(pos)
    n = len(pos)
    rows_t = None if rows is None else dev_i64(rows)
    m = n if rows_t is None else len(rows_t)
    div, curl, ddiv = (torch.empty(m, dtype=torch.float64, device=pos.device) for _ in range(3))
    off, idx = dev_i64(nb.offset), dev_i64(nb.index)
    ins = [dev_f64(vel), dev_f64(acc), dev_f64(mass, (n,)), dev_f64(h)]
    _call("nb_gradients", n, ptr(pos), *[ptr(a) for a in ins], ptr(off), ptr(idx), m,
          ptr(rows_t), KERNEL_IDS[kernel_name], ptr(div), ptr(curl), ptr(ddiv), stream())
    return Gradients(div, curl, ddiv)


def velocity_gradients_numba(pos, vel, mass, h, nb: Neighbours, kernel_name=DEFAULT_KERNEL,
                             rows=None, out=None) -> torch.Tensor:  # fmt: skip
    """sim/sph.py:827-846: fills ``out`` (N, 3, 3; zeros if not given) with the corrected
    gradients dv^i/dx^j of ``rows`` (default all) and returns it."""
    pos = dev_f64(pos)
    n = len(pos)
    rows_t = None if rows is None else dev_i64(rows)
    m = n if rows_t is None else len(rows_t)
    if out is None:
        out = torch.zeros((n, 3, 3), dtype=torch.float64, device=pos.device)
    elif out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous():
        raise ValueError("out must be a contiguous float64 CUDA tensor of shape (N, 3, 3)")
    off, idx = dev_i64(nb.offset), dev_i64(nb.index)
    ins = [dev_f64(vel), dev_f64(mass, (n,)), dev_f64(h)]
    _call("nb_velocity_gradients", n, ptr(pos), *[ptr(a) for a in ins], ptr(off), ptr(idx), m,
          ptr(rows_t), KERNEL_IDS[kernel_name], ptr(out), stream())
    return out


def disc_forces_numba(pos, vel, mass, h, rho, omega, c_s, alpha_av, nb: Neighbours,
                      kernel_name=DEFAULT_KERNEL, rows=None):  # fmt: skip
    """sim/sph.py:1120-1137: (acc (rows, 3), du/dt (rows,)) of the disc viscosity."""
    pos = dev_f64(pos)
    n = len(pos)
    rows_t = None if rows is None else dev_i64(rows)
    m = n if rows_t is None else len(rows_t)
    acc = torch.empty((m, 3), dtype=torch.float64, device=pos.device)
    dudt = torch.empty(m, dtype=torch.float64, device=pos.device)
    off, idx = dev_i64(nb.offset), dev_i64(nb.index)
    # every converted input stays referenced until the call returns
    ins = [dev_f64(vel), dev_f64(mass, (n,)), dev_f64(h), dev_f64(rho), dev_f64(omega),
           dev_f64(c_s)]  # fmt: skip
    _call("nb_disc_forces", n, ptr(pos), *[ptr(a) for a in ins], float(alpha_av), ptr(off),
          ptr(idx), m, ptr(rows_t), KERNEL_IDS[kernel_name], ptr(acc), ptr(dudt), stream())
    return acc, dudt


def glf_step_many(x, p, dt):
    """sim/integrator.py:188-198: one generalized-leapfrog step per particle; (x1, p1, iters).
    Raises GLFConvergenceError like the reference."""
    x = dev_f64(x)
    p = dev_f64(p)
    n = len(x)
    x1, p1 = torch.empty_like(x), torch.empty_like(p)
    it = torch.empty(n, dtype=torch.int64, device=x.device)
    if isinstance(dt, (int, float)) or (hasattr(dt, "ndim") and dt.ndim == 0):
        _call("nb_glf_step_many", n, ptr(x), ptr(p), None, float(dt), ptr(x1), ptr(p1), ptr(it),
              stream())  # fmt: skip
        return x1, p1, it
    else:
        dtt = dev_f64(dt, (n,))
        _call("nb_glf_step_many", n, ptr(x), ptr(p), ptr(dtt), 0.0, ptr(x1), ptr(p1), ptr(it),
              stream())  # fmt: skip
    return x1, p1, it


@dataclass
class Orbit:
    """A recorded orbit (sim/integrator.py:256-264): times, positions, momenta, iterations."""

    t: object
    x: object
    p: object
    iterations: object


def integrate_orbit(x0, p0, t_end, *, eta=None, dt=None, dt_max=4096.0, max_records=5_000_000):
    """sim/integrator.py:267-298: one particle from t = 0 to t_end with the generalized leapfrog
    on the integer tick timeline (adaptive quantized steps with eta, or fixed dt).  Returns NumPy
    arrays like the reference; raises GLFConvergenceError / ValueError like it."""
    import numpy as np

    if (eta is None) == (dt is None):
        raise ValueError("give exactly one of eta (adaptive) or dt (fixed)")
    if dt is not None:
        dt_max, eta = float(dt), 0.0
    tick = dt_max / 2.0**40
    n_end = int(round(t_end / tick))
    s0 = dev_f64(np.concatenate([np.asarray(x0, float), np.asarray(p0, float)]))
    d = s0.device
    t = torch.empty(max_records, dtype=torch.float64, device=d)
    s = torch.empty((max_records, 6), dtype=torch.float64, device=d)
    it = torch.empty(max_records, dtype=torch.int64, device=d)
    nrec = torch.empty(1, dtype=torch.int64, device=d)
    _call("nb_integrate_orbit", 1, ptr(s0), float(dt_max), float(eta), n_end, int(max_records),
          ptr(t), ptr(s), ptr(it), ptr(nrec), stream())  # fmt: skip
    m = int(nrec.item())
    if m == -5:
        raise ValueError(f"more than max_records={max_records} steps; raise max_records")
    if m < 0:
        msg = {-1: "stage 1 (p_half) did not converge in 10 iterations: time step too large",
               -2: "stage 2 (x1) did not converge in 10 iterations: time step too large",
               -3: "particle inside r = 2.5",
               -4: "time step would need more than 40 halvings of dt_max"}[m]  # fmt: skip
        raise GLFConvergenceError(msg)
    s = s[:m].cpu().numpy()
    return Orbit(t[:m].cpu().numpy(), s[:, :3].copy(), s[:, 3:].copy(), it[:m].cpu().numpy())


def gn_v_from_p(x, p):
    """sim/fastphys.py:35-42: v = A p + C (p.x) x."""
    x = dev_f64(x)
    p = dev_f64(p)
    v = torch.empty_like(x)
    _call("nb_gn_v_from_p", len(x), ptr(x), ptr(p), ptr(v), stream())
    return v


def gn_p_from_v(x, v):
    """physics/gravity.py:66-77: p = f v + g rdot x/r."""
    x = dev_f64(x)
    v = dev_f64(v)
    p = torch.empty_like(x)
    _call("nb_gn_p_from_v", len(x), ptr(x), ptr(v), ptr(p), stream())
    return p


def beta_cool(u, u_floor, dt, t_cool):
    """physics/cooling.py:33-40: u_floor + (u - u_floor) exp(-dt / t_cool)."""
    u = dev_f64(u)
    n = len(u)
    out = torch.empty_like(u)
    uf, dtt, tc = dev_f64(u_floor, (n,)), dev_f64(dt, (n,)), dev_f64(t_cool, (n,))
    _call("nb_beta_cool", n, ptr(u), ptr(uf), ptr(dtt), ptr(tc), ptr(out), stream())
    return out


def _eos_call(hc, rho, u, with_t):
    from .config import eos_fields

    rho = dev_f64(rho)
    u = dev_f64(u, rho.shape)
    prm = _lib.NbParams()
    prm.gamma = hc.gamma
    for k, v in eos_fields(hc).items():
        setattr(prm, k, v)
    n = len(rho)
    P, cs = torch.empty_like(rho), torch.empty_like(rho)
    T = torch.empty_like(rho) if with_t else None
    beta = torch.empty_like(rho) if with_t else None
    _call("nb_eos", n, ptr(rho), ptr(u), ctypes.byref(prm), ptr(P), ptr(cs),
          ptr(T) if with_t else None, ptr(beta) if with_t else None, stream())  # fmt: skip
    return P, cs, T, beta


def eos_state(cfg, rho, u):
    """sim/hydro.py:121-139 (ideal gas, radiation limit or gas + radiation): (P, c_s) in code
    units.  Raises FloatingPointError for u <= 0, ValueError for u outside the gas + radiation
    bracket [1, 1e13] K and RuntimeError if its temperature does not converge, as the reference."""
    if cfg.isothermal_cs is not None:
        raise NotImplementedError("isothermal equations of state are not part of the CUDA SPH path")
    P, cs, _, _ = _eos_call(cfg, rho, u, False)
    return P, cs


def gasrad_state(rho, u, gas_units=None):
    """gasrad_state_nb (sim/fastphys.py:93-107): (P [code], c_s [c], T [K], beta_gas) of gas +
    radiation in local thermodynamic equilibrium."""
    from .config import HydroConfig
    from .units import GasUnits

    hc = HydroConfig(eos="gasrad", gas_units=gas_units if gas_units is not None else GasUnits())
    return _eos_call(hc, rho, u, True)


def ledger_sums(x, p, u, mass) -> dict:
    """sim/coupled.py:261-270 sums on the device: energy sum m (H + u) (without radiated energy),
    sum m |H|, angular momentum, momentum, mass."""
    x, p, u, mass = dev_f64(x), dev_f64(p), dev_f64(u), dev_f64(mass)
    out = (ctypes.c_double * 9)()
    _call("nb_ledger", len(x), ptr(x), ptr(p), ptr(u), ptr(mass), out, stream())
    v = list(out)
    return {"energy": v[0], "abs_h": v[1], "angmom": v[2:5], "momentum": v[5:8], "mass": v[8]}

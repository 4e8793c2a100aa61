"""Shared-step API of the reference (sim/coupled.py:198-270) on the GPU.

``initialise``, ``step``, ``stable_dt``, ``ledger``, ``velocity`` keep the reference's names,
arguments and meaning; the state holds CUDA tensors (float64) and the whole step (list build or
reuse, density, EOS, forces, GN flow, cooling, kicks) runs in libnebula_b200.so.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import torch

from . import _lib
from .config import C_NORM, KERNEL_IDS, CoupledConfig, check_supported, eos_fields
from .cooling import brems_constants, floor_energy
from .device import ctx, dev_f64, ptr, stream, to_numpy
from . import ops


def make_params(cc: CoupledConfig, dt_max: float = 4096.0, limiter: bool = True,
                max_gap: int = 2) -> _lib.NbParams:  # fmt: skip
    """The flat parameter block of include/nebula_b200.h from the reference's configs."""
    check_supported(cc)
    hc = cc.hydro
    p = _lib.NbParams()
    kid = KERNEL_IDS[hc.kernel]
    p.kernel_id, p.cnorm, p.eta, p.tol, p.h_max, p.skin = kid, C_NORM[kid], hc.eta, 1e-4, hc.h_max, hc.skin
    p.gamma = hc.gamma
    p.viscosity, p.conductivity, p.cond_signal = int(hc.viscosity), int(hc.conductivity), int(hc.conductivity_signal)
    p.alpha_const, p.beta, p.alpha_u = hc.alpha_const, hc.beta, hc.alpha_u
    p.disc_alpha_av = hc.disc_alpha_av
    p.courant, p.c_force, p.eta_orb = hc.courant, hc.c_force, cc.eta_orb
    p.precision = 1 if hc.precision == "fp32" else 0
    if cc.cooling == "brems":
        bcst = brems_constants(hc.gamma, hc.gas_units, cc.t_floor)
        p.cooling = 2
        if cc.cooling_mlp is not None:  # the learned step, exact fallback inside
            p.cooling = 3
            p.mlp = cc.cooling_mlp.params
            cc.cooling_mlp.install()
        p.brems_tfac, p.brems_b, p.brems_kappa, p.brems_t_floor = bcst.tfac, bcst.b, bcst.kappa, bcst.t_floor
        p.u_floor = bcst.u_floor
    elif math.isfinite(cc.cooling_beta):
        p.cooling = 1
        p.cooling_beta = cc.cooling_beta
        p.u_floor = floor_energy(hc.gamma, cc.t_floor)
    p.dt_max, p.limiter, p.max_gap = dt_max, int(limiter), int(max_gap)
    # shock capturing of HydroConfig.shock() (sim/hydro.py:92-98)
    p.visc_switch = int(hc.viscosity and hc.switch)
    p.recon = int(hc.viscosity and hc.reconstruction)
    p.recon_closeness, p.recon_gate = int(bool(hc.recon_closeness)), int(hc.recon_gate)
    p.recon_eta_crit, p.recon_eta_fold = 1.0 / hc.eta, 0.2
    for k, v in eos_fields(hc).items():
        setattr(p, k, v)
    return p


@dataclass
class GasState:
    t: float
    x: torch.Tensor
    p: torch.Tensor
    u: torch.Tensor
    mass: torch.Tensor
    h: torch.Tensor
    alpha: torch.Tensor
    a_hydro: torch.Tensor = None
    dudt: torch.Tensor = None
    rho: torch.Tensor = None
    c_s: torch.Tensor = None
    vsig_max: torch.Tensor = None
    neighbour_cache: object = None
    e_radiated: float = 0.0
    visc_heating: torch.Tensor = None
    nu: torch.Tensor = None
    omega: torch.Tensor = None
    builds: int = 0
    reuses: int = 0
    particle_steps: int = 0
    _params: object = field(default=None, repr=False)

    def numpy(self) -> dict:
        return {k: to_numpy(v) for k, v in self.__dict__.items() if isinstance(v, torch.Tensor)}


def _state_struct(st) -> _lib.NbState:
    s = _lib.NbState()
    s.n = len(st.x)
    for name in ("x", "p", "u", "mass", "h", "alpha", "a_hydro", "dudt", "rho", "omega", "c_s",
                 "vsig_max", "nu", "visc_heating"):  # fmt: skip
        t = getattr(st, name, None)
        setattr(s, name, None if t is None else t.data_ptr())
    s.e_radiated = st.e_radiated
    s.builds, s.reuses, s.particle_steps = st.builds, st.reuses, st.particle_steps
    return s


def _pull(st, s: _lib.NbState) -> None:
    st.e_radiated = s.e_radiated
    st.builds, st.reuses, st.particle_steps = s.builds, s.reuses, s.particle_steps


def velocity(cfg: CoupledConfig, x, p):
    """sim/coupled.py:104-109: v = dH/dp (GN)."""
    return ops.gn_v_from_p(x, p)


def p_from_v(cfg: CoupledConfig, x, v):
    return ops.gn_p_from_v(x, v)


def _zeros(n, *shape):
    return torch.zeros((n, *shape), dtype=torch.float64, device=torch.device("cuda"))


def initialise(x, v, u, mass, h_guess, cfg: CoupledConfig, t: float = 0.0) -> GasState:
    """sim/coupled.py:198-210: state from positions and velocities (p computed from v), with
    density and forces evaluated."""
    prm = make_params(cfg)
    x = dev_f64(x)
    n = len(x)
    hc = cfg.hydro
    st = GasState(
        t=t, x=x.clone(), p=ops.gn_p_from_v(x, dev_f64(v)), u=dev_f64(u, (n,)).clone(),
        mass=dev_f64(mass, (n,)).clone(), h=dev_f64(h_guess, (n,)).clone(),
        alpha=torch.full((n,), hc.alpha_init if hc.switch else hc.alpha_const, dtype=torch.float64,
                         device=x.device),
        a_hydro=_zeros(n, 3), dudt=_zeros(n), rho=_zeros(n), c_s=_zeros(n), vsig_max=_zeros(n),
        visc_heating=_zeros(n), nu=_zeros(n), omega=torch.ones(n, dtype=torch.float64, device=x.device),
    )  # fmt: skip
    st._params = prm
    c = ctx()
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_coupled_initialise(c, ctypes.byref(s), ctypes.byref(prm), stream()))
    _pull(st, s)
    return st


def step(st: GasState, cfg: CoupledConfig, dt: float) -> GasState:
    """sim/coupled.py:238-258: one Strang-split kick-flow-kick step of size dt (in place; the
    state is also returned, as the reference returns its new state)."""
    prm = st._params if st._params is not None else make_params(cfg)
    c = ctx()
    s = _state_struct(st)
    _lib.check(c, _lib.lib().nb_coupled_step(c, ctypes.byref(s), ctypes.byref(prm), float(dt),
                                             stream()))  # fmt: skip
    _pull(st, s)
    st.t = st.t + dt
    return st


def stable_dt(st: GasState, cfg: CoupledConfig) -> float:
    """sim/coupled.py:213-226: min of the orbit, Courant, force and viscous criteria."""
    prm = st._params if st._params is not None else make_params(cfg)
    c = ctx()
    s = _state_struct(st)
    out = ctypes.c_double(0.0)
    _lib.check(c, _lib.lib().nb_coupled_stable_dt(c, ctypes.byref(s), ctypes.byref(prm),
                                                  ctypes.byref(out), stream()))  # fmt: skip
    return out.value


def ledger(st: GasState, cfg: CoupledConfig) -> dict:
    """sim/coupled.py:261-270: E = sum m (H + u) + E_radiated, angular momentum, sum m |H|."""
    s = ops.ledger_sums(st.x, st.p, st.u, st.mass)
    return {"energy": s["energy"] + st.e_radiated, "e_radiated": st.e_radiated,
            "abs_h": s["abs_h"], "angmom": s["angmom"], "momentum": s["momentum"],
            "mass": s["mass"]}  # fmt: skip

"""Cooling laws of the step: the reference's beta-cooling and optically thin bremsstrahlung.

beta-cooling is physics/cooling.py:23-40 (Gammie 2001).  Bremsstrahlung has no counterpart in
the reference: free-free emission eps = C_ff g_B T^(1/2) (1 + a T) n_e sum n_i Z_i^2 (Rybicki &
Lightman 1979, Eq. 5.15b, C_ff = 1.42e-27 erg cm^3 s^-1 K^-1/2, mean Gaunt factor g_B = 1.2, with
the relativistic factor 1 + 4.4e-10 T) for fully ionised gas of hydrogen fraction X = 0.7 and
metal fraction Z = 0.02, on the reference's ideal gas T = (gamma-1) mu m_p u / k and its 1e4 K
floor.  At fixed rho the temperature obeys dT/dt = -K rho T^(1/2) (1 + a T); arctan(sqrt(a T))
then falls linearly in time, which the kernel integrates exactly (the exact-integration idea of
Townsend 2009 for this Lambda(T)).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import units
from .device import ctx, dev_f64, ptr, stream
from . import _lib

C_FF = 1.42e-40  # W m^3 K^-1/2
GAUNT = 1.2
A_REL = 4.4e-10  # 1/K


@dataclass(frozen=True)
class BremsConstants:
    tfac: float  # K per code u
    b: float  # sqrt(A_REL)
    kappa: float  # fall of arctan(b sqrt T) per code density per code time
    u_floor: float  # code u at t_floor
    t_floor: float


def brems_constants(gamma: float = 5.0 / 3.0, gas_units: units.GasUnits = units.GasUnits(),
                    t_floor: float = 1.0e4) -> BremsConstants:  # fmt: skip
    length = gas_units.bh.length_m
    time = gas_units.bh.time_s
    rho_unit = gas_units.mass_kg_per_code / length**3
    tfac = (gamma - 1.0) * units.MU * units.M_P * units.C**2 / units.K_B
    comp = (1.0 + units.X_HYDROGEN) * (1.0 - units.Z_METALS) / 2.0
    k_si = (gamma - 1.0) * units.MU * units.M_P / units.K_B * C_FF * GAUNT * comp / units.M_P**2
    b = math.sqrt(A_REL)
    u_floor = units.K_B * t_floor / ((gamma - 1.0) * units.MU * units.M_P) / units.C**2
    return BremsConstants(tfac, b, 0.5 * b * k_si * rho_unit * time, u_floor, t_floor)


def floor_energy(gamma: float, t_floor: float) -> float:
    """sim/hydro.py:155-163 for eos="ideal": k T_floor / ((gamma-1) mu m_p) / c^2."""
    return units.K_B * t_floor / ((gamma - 1.0) * units.MU * units.M_P) / units.C**2


def brems_cool(u, rho, dt, consts: BremsConstants) -> torch.Tensor:
    """Exact bremsstrahlung cooling of u over dt at fixed rho (code units), on the GPU."""
    u = dev_f64(u)
    n = len(u)
    prm = _lib.NbParams()
    prm.brems_tfac, prm.brems_b, prm.brems_kappa = consts.tfac, consts.b, consts.kappa
    prm.u_floor, prm.brems_t_floor = consts.u_floor, consts.t_floor
    out = torch.empty_like(u)
    c = ctx()
    rho_t = dev_f64(rho, (n,))
    if isinstance(dt, (int, float)):
        st = _lib.lib().nb_brems_cool(c, n, ptr(u), ptr(rho_t), None, float(dt), prm, ptr(out),
                                      stream())  # fmt: skip
    else:
        dt_t = dev_f64(dt, (n,))
        st = _lib.lib().nb_brems_cool(c, n, ptr(u), ptr(rho_t), ptr(dt_t), 0.0, prm, ptr(out),
                                      stream())  # fmt: skip
    _lib.check(c, st)
    return out

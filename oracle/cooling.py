"""Cooling oracle (TEST INFRASTRUCTURE).

beta-cooling restates physics/cooling.py:23-40 (Gammie 2001; exact relaxation toward the floor).

Bremsstrahlung has NO counterpart in the reference (its only cooling law is beta-cooling), so this
part of the oracle is the build's own and is pinned by closed-form known answers in the tests, not
by reference output ("parity unpinned" against the reference for this law).  The law is the
optically thin free-free emissivity of Rybicki & Lightman (1979, Eq. 5.15b, with the relativistic
correction factor 1 + 4.4e-10 T widely used for hot plasma):

    eps = C_ff g_B T^(1/2) (1 + a T) n_e sum_i n_i Z_i^2,  C_ff = 1.42e-40 W m^3 K^-1/2,
    g_B = 1.2, a = 4.4e-10 K^-1, n_e sum n_i Z_i^2 = (rho/m_p)^2 (1+X)(1-Z)/2  (X = 0.7, Z = 0.02)

on an ideal gas T = (gamma-1) mu m_p u / k (the reference's temperature for eos="ideal",
sim/hydro.py:145-152) with the reference's 1e4 K floor (physics/cooling.py:19).  For fixed rho,
s = sqrt(T) obeys ds/dt = -(K rho/2)(1 + a s^2), so arctan(sqrt(a) s) falls linearly in time:
the integration is exact (Townsend 2009's exact-integration idea for this Lambda(T)).  Gas at or
below the floor does not cool; gas that would cool past it stops at the floor.
"""

from __future__ import annotations

import math

import numpy as np

C_FF = 1.42e-40  # W m^3 K^-1/2 (1.42e-27 erg cm^3 s^-1 K^-1/2)
GAUNT = 1.2
A_REL = 4.4e-10  # 1/K
G = 6.67430e-11
C = 299_792_458.0
M_SUN = 1.98847e30
K_B = 1.380649e-23
M_P = 1.67262192369e-27
MU = 0.6
X_H, Z_MET = 0.70, 0.02


def beta_cool(u, u_floor, dt, t_cool):
    """physics/cooling.py:33-40: u_floor + (u - u_floor) exp(-dt / t_cool)."""
    u = np.asarray(u, float)
    u_floor = np.asarray(u_floor, float)
    with np.errstate(divide="ignore"):
        decay = np.exp(-np.asarray(dt, float) / np.asarray(t_cool, float))
    return u_floor + (u - u_floor) * decay


def cooling_time(r, beta):
    """physics/cooling.py:23-30: beta / Omega_K, Omega_K = r^-1.5."""
    return beta / np.asarray(r, float) ** -1.5


def ideal_floor_energy(t_floor, gamma=5.0 / 3.0):
    """sim/hydro.py:155-163 for eos="ideal": k T_floor / ((gamma-1) mu m_p) / c^2."""
    return K_B * t_floor / ((gamma - 1.0) * MU * M_P) / C**2


def brems_constants(gamma=5.0 / 3.0, bh_mass_msun=4.3e6, gas_mass_msun=0.1, gas_mass_code=1.0,
                    t_floor=1.0e4):  # fmt: skip
    """(tfac, b, kappa, u_floor, T_floor): T = tfac u (code u), b = sqrt(a), and the fall of
    arctan(b sqrt(T)) per (code density x code time), kappa."""
    m_bh = bh_mass_msun * M_SUN
    length = G * m_bh / C**2
    time = G * m_bh / C**3
    rho_unit = gas_mass_msun * M_SUN / gas_mass_code / length**3  # kg/m^3 per code density
    tfac = (gamma - 1.0) * MU * M_P * C**2 / K_B
    comp = (1.0 + X_H) * (1.0 - Z_MET) / 2.0
    k_si = (gamma - 1.0) * MU * M_P / K_B * C_FF * GAUNT * comp / M_P**2  # dT/dt / (rho sqrt T ..)
    b = math.sqrt(A_REL)
    kappa = 0.5 * b * k_si * rho_unit * time
    return tfac, b, kappa, ideal_floor_energy(t_floor, gamma), t_floor


def brems_cool(u, rho, dt, consts):
    """Exact bremsstrahlung cooling over dt at fixed rho (code units): u after the step."""
    tfac, b, kappa, u_floor, t_floor = consts
    u = np.asarray(u, float)
    rho = np.broadcast_to(np.asarray(rho, float), u.shape)
    dt = np.broadcast_to(np.asarray(dt, float), u.shape)
    t0 = tfac * u
    th0 = np.arctan(b * np.sqrt(t0))
    th = th0 - kappa * rho * dt
    th_f = math.atan(b * math.sqrt(t_floor))
    ratio = np.tan(np.maximum(th, th_f)) / np.tan(th0)
    out = np.where(th <= th_f, u_floor, u * ratio * ratio)
    return np.where(t0 <= t_floor, u, out)


def brems_rate(u, rho, consts):
    """du/dt (code units, <= 0) of the same law, for the a-posteriori bracket checks."""
    tfac, b, kappa, u_floor, t_floor = consts
    t = tfac * np.asarray(u, float)
    return -2.0 * kappa / b * np.asarray(rho, float) * np.sqrt(t) * (1.0 + b * b * t) / tfac

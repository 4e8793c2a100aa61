"""CPU oracle of the equations of state (TEST INFRASTRUCTURE).

NumPy restatement (the T iteration in C, oracle.c) of sim/hydro.py:119-139 (eos_state), physics/eos.py:21-38 (ideal gas,
radiation limit) and the gas + radiation state of physics/eos.py:60-160 / sim/fastphys.py:45-107:
T from (rho, u) by Newton's method on log T inside a bisection bracket [1, 1e13] K narrowed every
iteration (tolerance 1e-12, at most 200 iterations), then P = rho k T/(mu m_p) + a T^4/3,
beta = P_gas/P, Gamma_1(beta) for gamma = 5/3 and c_s = sqrt(Gamma_1 P / rho).  Pinned bit for bit
to the reference's outputs in tests/golden/eos.npz.
"""

from __future__ import annotations

import numpy as np

from . import native

K_B = 1.380649e-23
M_P = 1.67262192369e-27
MU = 0.6
C = 299_792_458.0
A_RAD = 7.565733250033929e-16
T_MIN, T_MAX = 1.0, 1.0e13


def gasrad_temperature(rho_si, u_si):
    """T [K] of gas + radiation: physics/eos.py:110-144 / sim/fastphys.py:74-89, the iteration in
    C (``or_gasrad_temperature``) with the C library's exp, log and pow as the Numba kernel calls
    them.  Where f(T) rounds to a tiny non-zero value at the root, the reference's bracket test
    sends the iterate into bisection, so the result depends on the last bit of every operation."""
    rho = np.ravel(np.asarray(rho_si, float))
    u = np.ravel(np.broadcast_to(np.asarray(u_si, float), np.shape(rho_si)))
    a1 = 1.5 * K_B / (MU * M_P)
    if np.any(u < a1 * T_MIN + A_RAD * T_MIN**4 / rho) or np.any(u > a1 * T_MAX + A_RAD * T_MAX**4 / rho):
        raise ValueError("u outside the EOS bracket [1, 1e13] K")
    t, ok = native.gasrad_temperature(rho, u, a1, A_RAD)
    if not np.all(ok):
        raise RuntimeError("gas + radiation EOS: temperature did not converge")
    return t.reshape(np.shape(rho_si))


def gamma1(beta, gamma: float = 5.0 / 3.0):
    """physics/eos.py:101-106."""
    g = gamma - 1.0
    return beta + (4.0 - 3.0 * beta) ** 2 * g / (beta + 12.0 * g * (1.0 - beta))


def gasrad_state(rho_code, u_code, density_kg_m3: float):
    """(P [code], c_s [c], T [K], beta_gas) from code rho and u: sim/fastphys.py:92-107."""
    rho_code = np.asarray(rho_code, float)
    rho_si = rho_code * density_kg_m3
    t = gasrad_temperature(rho_si, np.asarray(u_code, float) * C**2)
    p_gas = rho_si * K_B * t / (MU * M_P)
    p_rad = A_RAD * t**4 / 3.0
    beta = p_gas / (p_gas + p_rad)
    p_code = (p_gas + p_rad) / (density_kg_m3 * C**2)
    return p_code, np.sqrt(gamma1(beta) * p_code / rho_code), t, beta


def eos_state(hc, rho, u):
    """sim/hydro.py:121-139 for the ideal gas, the radiation limit and gas + radiation."""
    rho = np.asarray(rho, float)
    u = np.asarray(u, float)
    if np.any(u <= 0):
        raise FloatingPointError(f"non-positive internal energy at {int(np.sum(u <= 0))} particles")
    if hc.eos == "ideal":
        return (hc.gamma - 1.0) * rho * u, np.sqrt(hc.gamma * (hc.gamma - 1.0) * u)
    if hc.eos == "radiation":
        return rho * u / 3.0, np.sqrt(4.0 * u / 9.0)
    if hc.eos == "gasrad":
        p, cs, _, _ = gasrad_state(rho, u, hc.gas_units.density_kg_m3)
        return p, cs
    raise ValueError(f"unknown equation of state {hc.eos!r}")

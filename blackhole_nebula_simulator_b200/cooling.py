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

import ctypes
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


# --------------------------------------------------------------------------- learned cooling
NPARAM = 8641  # 3 -> 64 -> 64 -> 64 -> 1


@dataclass(frozen=True)
class Hull:
    """Training hull of the network: log10 rho [g/cm^3], log10 T [K], log10 dt [s]."""

    lrho: tuple = (-14.0, -6.0)
    lt: tuple = (4.0, 10.0)
    ldt: tuple = (-2.0, 3.0)


def mlp_params(gamma: float = 5.0 / 3.0, gas_units: units.GasUnits = units.GasUnits(),
               t_floor: float = 1.0e4, hull: Hull = Hull(), check_tol: float = 5.0e-4,
               judge: int = 0) -> _lib.NbMlpParams:  # fmt: skip
    """The network's parameter block: the bremsstrahlung law, the unit conversions of its inputs,
    the hull, the a-posteriori tolerance tol (fraction of u; an accepted step is within 2 tol of
    the exact integrator) and the judge stride (0: off)."""
    c = brems_constants(gamma, gas_units, t_floor)
    p = _lib.NbMlpParams()
    p.tfac, p.b, p.kappa, p.u_floor, p.t_floor = c.tfac, c.b, c.kappa, c.u_floor, c.t_floor
    p.rho_unit_cgs = gas_units.density_kg_m3 * 1.0e-3
    p.t_unit_s = gas_units.bh.time_s
    p.lrho_lo, p.lrho_hi = hull.lrho
    p.lt_lo, p.lt_hi = hull.lt
    p.ldt_lo, p.ldt_hi = hull.ldt
    p.check_tol, p.judge = check_tol, judge
    return p


@dataclass
class CoolingNetwork:
    """A trained network (float32 weights on the device) and the parameter block it was trained
    with; pass it as CoupledConfig(cooling="brems", cooling_mlp=net)."""

    weights: torch.Tensor
    params: object
    loss_history: list = None

    def install(self) -> None:
        c = ctx()
        _lib.check(c, _lib.lib().nb_mlp_weights(c, None, ptr(self.weights), stream()))


def train_network(n_samples: int = 16 * 2**20, batch: int = 32768, epochs: int = 40,
                  lr: float = 3.0e-3, seed: int = 2026, params=None) -> CoolingNetwork:  # fmt: skip
    """Train the cooling network on the GPU with the library's own kernels: n_samples
    log-uniform samples labelled by the exact integrator, Adam with a cosine learning rate."""
    prm = params if params is not None else mlp_params()
    c = ctx()
    hist = (ctypes.c_float * epochs)()
    _lib.check(c, _lib.lib().nb_mlp_train(c, prm, int(n_samples), int(batch), int(epochs),
                                          float(lr), int(seed), hist, stream()))  # fmt: skip
    w = torch.empty(NPARAM, dtype=torch.float32, device=torch.device("cuda"))
    _lib.check(c, _lib.lib().nb_mlp_weights(c, ptr(w), None, stream()))
    return CoolingNetwork(w, prm, list(hist))


def load_network(path: str, params=None) -> CoolingNetwork:
    import numpy as np

    w = torch.as_tensor(np.load(path).astype(np.float32), device=torch.device("cuda"))
    return CoolingNetwork(w, params if params is not None else mlp_params())


def mlp_cool(u, rho, dt, net: CoolingNetwork, params=None):
    """Cooling by the network with exact fallback: (u_new, mode) with mode 0 exact / no cooling,
    1 network, 2 fallback."""
    net.install()
    prm = params if params is not None else net.params
    u = dev_f64(u)
    n = len(u)
    rho_t = dev_f64(rho, (n,))
    out = torch.empty_like(u)
    mode = torch.empty(n, dtype=torch.int8, device=u.device)
    c = ctx()
    if isinstance(dt, (int, float)):
        st = _lib.lib().nb_mlp_cool(c, n, ptr(u), ptr(rho_t), None, float(dt), prm, ptr(out),
                                    ptr(mode), stream())  # fmt: skip
    else:
        dt_t = dev_f64(dt, (n,))
        st = _lib.lib().nb_mlp_cool(c, n, ptr(u), ptr(rho_t), ptr(dt_t), 0.0, prm, ptr(out),
                                    ptr(mode), stream())  # fmt: skip
    _lib.check(c, st)
    return out, mode


def mlp_stats(reset: bool = False) -> dict:
    """Judge statistics of the network against the exact integrator since the last reset."""
    c = ctx()
    out = (ctypes.c_double * 5)()
    _lib.check(c, _lib.lib().nb_mlp_stats(c, out, int(reset)))
    return {"max_err": out[0], "rms_err": out[1], "judged": int(out[2]), "network": int(out[3]),
            "fallback": int(out[4])}  # fmt: skip


def main(argv=None) -> None:
    """python -m blackhole_nebula_simulator_b200.cooling OUT.npy [n_samples epochs]: train the
    network on the GPU and save its float32 weights."""
    import sys

    import numpy as np

    args = sys.argv[1:] if argv is None else argv
    out = args[0]
    n = int(args[1]) if len(args) > 1 else 16 * 2**20
    epochs = int(args[2]) if len(args) > 2 else 40
    net = train_network(n_samples=n, epochs=epochs)
    np.save(out, net.weights.cpu().numpy())
    print(f"trained on {n} samples, {epochs} epochs; last-batch loss per epoch: "
          + " ".join(f"{v:.3g}" for v in net.loss_history))


if __name__ == "__main__":
    main()

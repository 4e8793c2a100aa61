"""Run configuration for the SPH step: the reference's frozen dataclasses, field for field.

The field names, meanings and defaults are those of the reference (sim/hydro.py:53-98
``HydroConfig``, sim/sph.py:409-430 ``ShockCapturing``, sim/coupled.py:62-75 ``CoupledConfig``,
sim/blocks.py:83-100 ``BlockConfig``), so a driver written against the reference builds the same
objects here.  Two fields are added to ``CoupledConfig`` for the bremsstrahlung cooling and its
learned replacement (``cooling``, ``cooling_mlp``) and one to ``HydroConfig`` for the pair
arithmetic (``precision``); their defaults leave the reference behaviour unchanged.

Options of the reference that the CUDA path does not implement are rejected with
``NotImplementedError`` by ``check_supported`` instead of being ignored.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

from . import units

COND_PRESSURE = 0  # v^u_sig = sqrt(|P_a - P_b| / rho_ab)
COND_VELOCITY = 1  # v^u_sig = |v_ab . r_hat_ab|
GATE_BOTH, GATE_PUBLISHED, GATE_MINMOD = 0, 1, 2

BETA_AV = 2.0
ALPHA_U = 1.0
ALPHA_U_MAGMA2 = 0.05
H_MAX_HOLE = 200.0  # smoothing-length cap with the hole (sim/coupled.py:59)
T_FLOOR = 1.0e4  # K (physics/cooling.py:19)

KERNEL_IDS = {"cubic": 0, "wendland_c4": 1}
C_NORM = (1.0 / math.pi, 495.0 / (256.0 * math.pi))  # physics/kernels.py:94-95
HFACT = {"cubic": 1.2, "wendland_c4": 1.6}
DEFAULT_KERNEL = "wendland_c4"  # physics/kernels.py:101-102
DEFAULT_ETA = 1.6


@dataclass(frozen=True)
class ShockCapturing:
    beta: float = BETA_AV
    alpha_u: float = ALPHA_U
    conductivity_signal: int = COND_PRESSURE
    reconstruction: bool = False
    closeness: bool = True
    eta_crit: float = 1.0 / DEFAULT_ETA
    eta_fold: float = 0.2
    recon_gate: int = GATE_MINMOD


@dataclass(frozen=True)
class HydroConfig:
    gamma: float = 5.0 / 3.0
    isothermal_cs: float | None = None
    iso_r0: float | None = None
    iso_q: float = 0.75
    eos: str = "ideal"
    gas_units: units.GasUnits = units.GasUnits()
    kernel: str = DEFAULT_KERNEL
    eta: float = DEFAULT_ETA
    box: tuple | None = None
    h_max: float = math.inf
    courant: float = 0.3
    skin: float = 1.4
    c_force: float = 0.25
    viscosity: bool = True
    conductivity: bool = True
    switch: bool = True
    alpha_const: float = 1.0
    alpha_init: float = 0.0
    beta: float = BETA_AV
    alpha_u: float = ALPHA_U
    conductivity_signal: int = COND_PRESSURE
    reconstruction: bool = True
    recon_closeness: bool = True
    recon_gate: int = GATE_MINMOD
    ns_nu: float = 0.0
    ns_alpha: float = 0.0
    disc_alpha_av: float = 0.0
    # pair arithmetic of the CUDA path: "fp64" (every pair term in double) or "fp32" (cell-relative
    # float offsets, Kahan-compensated sums; lists, drift, gravity and ledgers stay double)
    precision: str = "fp64"

    def shock(self) -> ShockCapturing:
        return ShockCapturing(
            self.beta, self.alpha_u, self.conductivity_signal,
            reconstruction=self.reconstruction and self.viscosity,
            closeness=self.recon_closeness, eta_crit=1.0 / self.eta, recon_gate=self.recon_gate,
        )  # fmt: skip


@dataclass(frozen=True)
class CoupledConfig:
    hydro: HydroConfig = HydroConfig(
        conductivity_signal=COND_VELOCITY, alpha_u=ALPHA_U_MAGMA2, h_max=H_MAX_HOLE
    )
    hole: bool = True
    eta_orb: float = 0.00125
    wrong_coupling: bool = False
    gravity: str = "gn"
    cooling_beta: float = math.inf
    t_floor: float = T_FLOOR
    # optically thin bremsstrahlung cooling (cooling.py): "none" or "brems"; with cooling_mlp the
    # learned network replaces the exact integrator where its checks pass
    cooling: str = "none"
    cooling_mlp: object = None


@dataclass(frozen=True)
class BlockConfig:
    coupled: CoupledConfig = CoupledConfig()
    dt_max: float = 4096.0
    limiter: bool = True
    max_gap: int = 2
    hydro: bool = True
    r_acc: float | None = None
    r_escape: float | None = None
    respa: bool = False
    respa_eta: float = 0.05
    removal_sync: bool = True


# equations of state of sim/hydro.py:121-139 and their ids in nb_params.eos
EOS_IDS = {"ideal": 0, "gasrad": 1, "radiation": 2}


def eos_fields(hc) -> dict:
    """The nb_params EOS fields of a HydroConfig (gas + radiation in SI inside the T-solve)."""
    return dict(eos=EOS_IDS[hc.eos], eos_rho_si=hc.gas_units.density_kg_m3, eos_u_si=units.C**2,
                eos_a1=1.5 * units.K_B / (units.MU * units.M_P), eos_a_rad=units.A_RAD)  # fmt: skip


def check_supported(cc: CoupledConfig) -> None:
    """Raise NotImplementedError for reference options outside the CUDA path."""
    hc = cc.hydro
    bad = []
    if hc.box is not None:
        bad.append("periodic box")
    if hc.isothermal_cs is not None:
        bad.append("isothermal equation of state")
    if hc.eos not in EOS_IDS:
        raise ValueError(f"unknown equation of state {hc.eos!r}")
    cooling_on = cc.cooling == "brems" or math.isfinite(cc.cooling_beta)
    if hc.eos != "ideal" and cooling_on:
        bad.append(f"cooling with eos={hc.eos!r} (the floor energy then depends on rho)")
    if hc.recon_gate not in (GATE_BOTH, GATE_PUBLISHED, GATE_MINMOD):
        raise ValueError(f"unknown reconstruction gate {hc.recon_gate!r}")
    if hc.ns_nu > 0 or hc.ns_alpha > 0:
        bad.append("Navier-Stokes viscosity (ns_nu / ns_alpha)")
    if cc.wrong_coupling:
        bad.append("wrong_coupling")
    if cc.gravity != "gn" or not cc.hole:
        bad.append("gravity other than the GN hole")
    if hc.kernel not in KERNEL_IDS:
        raise ValueError(f"unknown kernel {hc.kernel!r}; choose from {sorted(KERNEL_IDS)}")
    if hc.precision not in ("fp64", "fp32"):
        raise ValueError(f"precision must be 'fp64' or 'fp32', not {hc.precision!r}")
    if cc.cooling not in ("none", "brems"):
        raise ValueError(f"cooling must be 'none' or 'brems', not {cc.cooling!r}")
    if cc.cooling == "brems" and math.isfinite(cc.cooling_beta):
        raise ValueError("choose one cooling law: beta-cooling or bremsstrahlung")
    if bad:
        raise NotImplementedError("not in the CUDA SPH path: " + ", ".join(bad))

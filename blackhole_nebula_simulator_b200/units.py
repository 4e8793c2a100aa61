"""Physical constants and code units (G = c = M_bh = 1) used by the SPH step.

The constants are CODATA 2018 values and the unit definitions are the reference's
(units.py:18-39, 52-133): length GM/c^2, time GM/c^3, specific energy c^2, and a separate gas
mass scale (0.1 M_sun of gas per code mass unit) that fixes the physical density.
"""

from __future__ import annotations

from dataclasses import dataclass

G = 6.67430e-11  # m^3 kg^-1 s^-2
C = 299_792_458.0  # m/s
M_SUN = 1.98847e30  # kg
K_B = 1.380649e-23  # J/K
M_P = 1.67262192369e-27  # kg
MU = 0.6  # mean molecular weight, fully ionised solar gas
A_RAD = 7.565733250033929e-16  # radiation constant 4 sigma / c [J m^-3 K^-4]
X_HYDROGEN = 0.70
Z_METALS = 0.02
SGR_A_MASS_MSUN = 4.3e6
CLOUD_MASS_MSUN = 0.1


@dataclass(frozen=True)
class BlackHoleUnits:
    mass_msun: float = SGR_A_MASS_MSUN

    @property
    def mass_kg(self) -> float:
        return self.mass_msun * M_SUN

    @property
    def length_m(self) -> float:
        return G * self.mass_kg / C**2

    @property
    def time_s(self) -> float:
        return G * self.mass_kg / C**3


@dataclass(frozen=True)
class GasUnits:
    bh: BlackHoleUnits = BlackHoleUnits()
    cloud_mass_msun: float = CLOUD_MASS_MSUN
    cloud_mass_code: float = 1.0

    @property
    def mass_kg_per_code(self) -> float:
        return self.cloud_mass_msun * M_SUN / self.cloud_mass_code

    @property
    def density_kg_m3(self) -> float:
        return self.mass_kg_per_code / self.bh.length_m**3

    def density_to_si(self, rho_code):
        return rho_code * self.density_kg_m3

    def density_from_si(self, rho_si):
        return rho_si / self.density_kg_m3


def specific_energy_to_si(u_code):
    return u_code * C**2


def specific_energy_from_si(u_si):
    return u_si / C**2


def gas_temperature_from_u(u_code, gamma: float = 5.0 / 3.0):
    """Ideal-gas temperature (K) of code specific energy u: T = (gamma-1) mu m_p u c^2 / k."""
    return (gamma - 1.0) * MU * M_P * specific_energy_to_si(u_code) / K_B


def gas_u_from_temperature(t_kelvin, gamma: float = 5.0 / 3.0):
    """Code specific energy of an ideal gas at T: u = k T / ((gamma-1) mu m_p) / c^2."""
    return specific_energy_from_si(K_B * t_kelvin / ((gamma - 1.0) * MU * M_P))

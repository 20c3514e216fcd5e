"""Physical constants and particle species.

CODATA 2018 values, as src/utility/constants.jl:1-20 of the reference takes
them from PhysicalConstants.jl, plus the Earth radius and dipole moment.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

qe = -1.602176634e-19          # electron charge [C]
me = 9.1093837015e-31          # electron mass [kg]
qi = 1.602176634e-19           # proton charge [C]
mi = 1.67262192369e-27         # proton mass [kg]
c = 299792458.0                # speed of light [m/s]
mu0 = 1.25663706212e-6         # vacuum permeability [H/m]
eps0 = 8.8541878128e-12        # vacuum permittivity [F/m]
kB = 1.380649e-23              # Boltzmann constant [J/K]
Re = 6371.0e3                  # Earth radius [m]
BMoment_Earth = (0.0, 0.0, -7.94e22)  # Earth dipole moment [A m^2]
eV = qi                        # electron volt [J]
MU0_OVER_4PI = mu0 / (4.0 * math.pi)


@dataclass(frozen=True)
class Species:
    """Particle species with mass `m` [kg] and charge `q` [C] (src/types.jl:18-21)."""

    m: float
    q: float


Proton = Species(mi, qi)
Electron = Species(me, qe)


def Ion(m: float = 1, q: float = 1) -> Species:
    """Ion with mass number `m` and charge number `q` (constants.jl:19-20)."""
    return Species(m * mi, q * qi)


SpeciesDict = {
    "H+": Proton,
    "Proton": Proton,
    "e-": Electron,
    "Electron": Electron,
    "O+": Ion(16, 1),
    "He+": Ion(4, 1),
    "O2+": Ion(32, 1),
    "CO2+": Ion(44, 1),
}

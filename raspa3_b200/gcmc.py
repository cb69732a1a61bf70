"""Rigid adsorbate components and thermodynamic conditions of the GCMC workloads.

Units follow RASPA3's System constructor (src/raspakit/system.cpp:96-98): beta = 1 / (KB T) with KB in internal energy
units per Kelvin, pressure = P[Pa] / PressureConversionFactor. A component's body frame is centred on its centre of
mass, the point the rotation move turns the molecule about (mc_moves/component/rotation.cpp).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .forcefield import KB, PRESSURE_CONVERSION_FACTOR, ForceField


@dataclass
class RigidComponent:
    name: str
    names: tuple[str, ...]
    offsets: np.ndarray  # (n, 3) body frame relative to the centre of mass
    masses: np.ndarray
    starting_bead: int

    @property
    def n_atoms(self) -> int:
        return len(self.names)

    def types(self, ff: ForceField) -> np.ndarray:
        return np.array([ff.index(n) for n in self.names], dtype=np.int32)

    def charges(self, ff: ForceField) -> np.ndarray:
        return np.array([ff.pseudo_atoms[ff.index(n)].charge for n in self.names])


def _centred(offsets, masses):
    offsets = np.asarray(offsets, dtype=np.float64)
    masses = np.asarray(masses, dtype=np.float64)
    com = (masses[:, None] * offsets).sum(0) / masses.sum()
    return offsets - com


def co2_component(bond: float = 1.16) -> RigidComponent:
    """Rigid 3-site CO2 (C-O 1.16 A), O-C-O order as Component::makeCO2 (component.cpp:2304-2329); CBMC grows it from
    the central C atom."""
    m = np.array([15.9994, 12.0, 15.9994])
    return RigidComponent("CO2", ("O_co2", "C_co2", "O_co2"),
                          _centred([(0, 0, bond), (0, 0, 0), (0, 0, -bond)], m), m, 1)


def n2_component(bond: float = 1.10) -> RigidComponent:
    """3-site N2: N-N 1.10 A with the massless charge site N_com at the centre; grown from atom 0 (an N), the
    reference's default starting bead (Component::startingBead, component.ixx:195)."""
    m = np.array([14.00674, 0.0, 14.00674])
    return RigidComponent("N2", ("N_n2", "N_com", "N_n2"),
                          _centred([(0, 0, 0.5 * bond), (0, 0, 0), (0, 0, -0.5 * bond)], m), m, 0)


def methane_component() -> RigidComponent:
    """United-atom methane (Component::makeMethane, component.cpp:2290-2302)."""
    return RigidComponent("methane", ("CH4",), np.zeros((1, 3)), np.array([16.04246]), 0)


def beta_of(temperature: float) -> float:
    return 1.0 / (KB * temperature)


def fugacity_of(pressure_pa: float) -> float:
    """Ideal-gas fugacity (fugacity coefficient 1) in internal pressure units."""
    return pressure_pa / PRESSURE_CONVERSION_FACTOR

"""Flexible united-atom alkane chains and the batched many-system CBMC workload.

A chain is the reference Component of a linear molecule with fixed bonds, harmonic bends and TraPPE torsions, grown
from bead 0 by configurational-bias Monte Carlo (cbmc/flexible_molecules/insertion.cpp). TraPPE-UA parameters
(Martin & Siepmann, J. Phys. Chem. B 102, 2569 (1998)): CH3 98 K / 3.75 A, CH2 46 K / 3.95 A, 1.54 A bonds,
k_theta = 62500 K/rad^2 around 114 degrees, torsion p0..p3 = 0, 355.03, -68.19, 791.32 K.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from .forcefield import KELVIN_TO_ENERGY, ForceField, box_struct, perpendicular_widths
from .synthetic import batched_frameworks, replicate, synthetic_forcefield

TRAPPE_TORSION_K = (0.0, 355.03, -68.19, 791.32)


@dataclass
class AlkaneChain:
    n_beads: int
    bond_length: float = 1.54
    bend_k_kelvin: float = 62500.0
    bend_theta0_deg: float = 114.0
    torsion_kelvin: tuple = TRAPPE_TORSION_K
    n_first: int = 10
    n_directions: int = 10
    n_torsion: int = 100
    n_moves_per_open_bead: int = 150
    type_names: list = field(default_factory=list)

    def __post_init__(self):
        if not self.type_names:
            self.type_names = ["CH3"] + ["CH2"] * (self.n_beads - 2) + ["CH3"] if self.n_beads > 1 else ["CH4"]

    def types(self, ff: ForceField) -> list[int]:
        return [ff.index(n) for n in self.type_names]


class RgAlkaneChain(ctypes.Structure):
    _fields_ = [("n_beads", ctypes.c_int32), ("types", ctypes.c_int32 * 8), ("bond_length", ctypes.c_double),
                ("bend_k", ctypes.c_double), ("bend_theta0", ctypes.c_double), ("torsion", ctypes.c_double * 4),
                ("n_first_bead_trials", ctypes.c_int32), ("n_trial_directions", ctypes.c_int32),
                ("n_torsion_trials", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def chain_struct(chain: AlkaneChain, ff: ForceField) -> RgAlkaneChain:
    c = RgAlkaneChain()
    c.n_beads = chain.n_beads
    for i, t in enumerate(chain.types(ff)):
        c.types[i] = t
    c.bond_length = chain.bond_length
    c.bend_k = chain.bend_k_kelvin * KELVIN_TO_ENERGY
    c.bend_theta0 = math.radians(chain.bend_theta0_deg)
    for k in range(4):
        c.torsion[k] = chain.torsion_kelvin[k] * KELVIN_TO_ENERGY
    c.n_first_bead_trials = chain.n_first
    c.n_trial_directions = chain.n_directions
    c.n_torsion_trials = chain.n_torsion
    return c


@dataclass
class AlkaneSystem:
    """One system of the batch: simulation box, its framework atoms, the chain and the thermodynamic state."""
    cell: np.ndarray
    framework: np.ndarray
    chain: AlkaneChain
    beta: float
    fugacity: float
    w_ig: float = 1.0
    max_molecules: int = 64
    max_translation: float = 1.0
    p_translation: float = 1.0
    p_swap: float = 1.0


def replicate_for_cutoff(cell, atoms, cutoff: float = 12.0):
    """SimulationBox::smallestNumberOfUnitCellsForMinimumImagesConvention (simulationbox.cpp:150-156)."""
    w = perpendicular_widths(cell)
    reps = tuple(int(math.ceil(2.0 * cutoff / float(x))) for x in w)
    scell, satoms = replicate(cell, atoms, reps)
    return scell, satoms, reps


def alkane_forcefield(rc: float = 12.0) -> ForceField:
    """The synthetic framework force field without charges (T: no LJ, O 89.6 K / 3.0 A) plus CH3 / CH2, shifted."""
    return synthetic_forcefield(rc=rc, charges=False)


ALKANE_FRAMEWORK_DENSITY = 0.025  # framework atoms per cubic Angstrom


def alkane_batch_systems(ff: ForceField, n_systems: int = 64, seed: int = 1234, temperature: float = 300.0,
                    pressure: float = 1e5, cutoff: float = 12.0, max_molecules: int = 64, chain_lengths=(4, 8),
                    trials=None, density: float = ALKANE_FRAMEWORK_DENSITY):
    """The batched-CBMC workload: synthetic cells with lengths uniform in [12, 40] A and 96-1536 atoms
    (batched_frameworks; the count is density x volume clipped to that range), each replicated for the minimum image of
    the cutoff, with a chain of 4-8 beads drawn per system. The density of 0.025 per cubic Angstrom leaves channels
    for CH2/CH3 beads between randomly placed atoms (at the 0.054 atoms per cubic Angstrom of the 20.0 x 19.9 x 13.4 A cell they are closed).
    trials: optional (n_first, n_directions) per system for uneven trial counts (default 10 / 10)."""
    from .gcmc import beta_of, fugacity_of

    rng = np.random.default_rng(seed + 7)
    systems = []
    for s, (cell, atoms) in enumerate(batched_frameworks(ff, n_systems=n_systems, seed=seed, density=density)):
        scell, satoms, _ = replicate_for_cutoff(cell, atoms, cutoff)
        nb = int(rng.integers(chain_lengths[0], chain_lengths[1] + 1))
        nf, nd = (10, 10) if trials is None else trials[s]
        systems.append(AlkaneSystem(cell=scell, framework=satoms, chain=AlkaneChain(nb, n_first=nf, n_directions=nd),
                                    beta=beta_of(temperature), fugacity=fugacity_of(pressure),
                                    max_molecules=max_molecules))
    return systems

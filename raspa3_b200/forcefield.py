"""Force-field tables, unit constants and the atom record shared by the host code and the C-ABI.

The pair table follows RASPA3's ``ForceField``:

* Lorentz-Berthelot mixing of the self-interaction parameters: ``src/raspakit/forcefield/forcefield.cpp:924-960``.
* The potential shift at the pair cutoff: ``forcefield.cpp:1016-1051`` and
  ``forcefield/vdwparameters.cpp:211-223``.
* Epsilon converted from Kelvin to internal units on construction:
  ``forcefield/vdwparameters.ixx:114``.

The unit constants are computed with the same expressions as ``src/raspakit/units.cpp:14-98`` from the base
constants of ``src/foundationkit/units.ixx:29-55``, so every value is the same IEEE double the reference uses.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

# ---- units (src/foundationkit/units.ixx:29-55, src/raspakit/units.cpp:14-98) ----
ANGSTROM = 1e-10
PICO_SECOND = 1e-12
ATOMIC_MASS_UNIT = 1.6605402e-27
ELECTRONIC_CHARGE_UNIT = 1.60217733e-19
MOLAR_GAS_CONSTANT = 8.314464919
BOLTZMANN_CONSTANT = 1.380650324e-23
AVOGADRO_CONSTANT = 6.0221419947e23
DIELECTRIC_CONSTANT_VACUUM = 8.8541878176e-12

ENERGY_CONVERSION_FACTOR = ATOMIC_MASS_UNIT * ANGSTROM * ANGSTROM / (PICO_SECOND * PICO_SECOND)
ENERGY_TO_KELVIN = ENERGY_CONVERSION_FACTOR * AVOGADRO_CONSTANT / MOLAR_GAS_CONSTANT
KELVIN_TO_ENERGY = MOLAR_GAS_CONSTANT / (ENERGY_CONVERSION_FACTOR * AVOGADRO_CONSTANT)
COULOMBIC_CONVERSION_FACTOR = ELECTRONIC_CHARGE_UNIT * ELECTRONIC_CHARGE_UNIT / (
    4.0 * math.pi * DIELECTRIC_CONSTANT_VACUUM * ANGSTROM * ENERGY_CONVERSION_FACTOR)
# Boltzmann constant in internal energy units per Kelvin (units.cpp: KB).
KB = BOLTZMANN_CONSTANT / ENERGY_CONVERSION_FACTOR
PRESSURE_CONVERSION_FACTOR = ATOMIC_MASS_UNIT / (ANGSTROM * PICO_SECOND * PICO_SECOND)

# ---- the 64-byte atom record, layout-identical to RASPA3's Atom (src/raspakit/atom.ixx:28-39) ----
ATOM_DTYPE = np.dtype([
    ("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("w", "<f8"),
    ("charge", "<f8"), ("scaling_vdw", "<f8"), ("scaling_coulomb", "<f8"),
    ("molecule_id", "<u4"), ("type", "<u2"), ("component_id", "u1"), ("group_fractional", "u1"),
])
assert ATOM_DTYPE.itemsize == 64


def make_atoms(positions, types, charges, molecule_ids=None, scaling_vdw=None, scaling_coulomb=None,
               group_ids=None, fractional=None, component_ids=None) -> np.ndarray:
    """Pack per-atom arrays into the 64-byte record array passed through the C-ABI."""
    positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    n = positions.shape[0]
    a = np.zeros(n, dtype=ATOM_DTYPE)
    a["x"], a["y"], a["z"] = positions[:, 0], positions[:, 1], positions[:, 2]
    a["charge"] = np.broadcast_to(np.asarray(charges, dtype=np.float64), (n,))
    a["type"] = np.broadcast_to(np.asarray(types), (n,))
    a["scaling_vdw"] = 1.0 if scaling_vdw is None else scaling_vdw
    a["scaling_coulomb"] = 1.0 if scaling_coulomb is None else scaling_coulomb
    if molecule_ids is not None:
        a["molecule_id"] = molecule_ids
    if component_ids is not None:
        a["component_id"] = component_ids
    g = np.zeros(n, dtype=np.uint8) if group_ids is None else np.asarray(group_ids, dtype=np.uint8)
    f = np.zeros(n, dtype=np.uint8) if fractional is None else np.asarray(fractional, dtype=np.uint8)
    a["group_fractional"] = (g & 0x0F) | ((f & 0x0F) << 4)
    return a


def positions_of(atoms: np.ndarray) -> np.ndarray:
    return np.stack([atoms["x"], atoms["y"], atoms["z"]], axis=1)


def lambda_scaling(lam: float) -> tuple[float, float]:
    """Scaling::scalingVDW / scalingCoulomb (src/raspakit/scaling.ixx:7-25)."""
    t = 2.0 * lam
    it = 1.0 - t
    svdw = (t * t) / (t * t + it * it) if lam < 0.5 else 1.0
    t = 2.0 * (lam - 0.5)
    it = 1.0 - t
    scoul = (t * t) / (t * t + it * it) if lam > 0.5 else 0.0
    return svdw, scoul


@dataclass
class PseudoAtom:
    name: str
    framework: bool
    epsilon_k: float  # Kelvin
    sigma: float      # Angstrom
    charge: float = 0.0
    mass: float = 0.0
    lj: bool = True


@dataclass
class ForceField:
    """Mixed, shifted pair table in internal units plus the scalar parameters of the three paths."""

    pseudo_atoms: list[PseudoAtom]
    cutoff_framework_vdw: float = 12.0
    cutoff_molecule_vdw: float = 12.0
    cutoff_coulomb: float = 12.0
    shifted: bool = True
    ewald_alpha: float = 0.265058
    kmax: tuple[int, int, int] = (8, 8, 8)
    # Integer k-sphere bound kx^2+ky^2+kz^2 <= this; 2**64-1 means the full half-box (manual EwaldParameters,
    # forcefield.cpp:388-418); the automatic setting uses max(kmax)^2 (forcefield.cpp:1415-1438).
    recip_int_cutoff_sq: int = (1 << 64) - 1
    recip_cutoff_sq: float = float(np.finfo(np.float64).max)
    overlap_criteria: float = 1e6
    use_charge: bool = True
    omit_inter: bool = False
    epsilon: np.ndarray = field(init=False)
    sigma: np.ndarray = field(init=False)
    shift: np.ndarray = field(init=False)
    lj: np.ndarray = field(init=False)

    def __post_init__(self):
        n = len(self.pseudo_atoms)
        eps = np.zeros((n, n))
        sig = np.ones((n, n))
        lj = np.zeros((n, n), dtype=np.int32)
        for i, p in enumerate(self.pseudo_atoms):
            eps[i, i] = p.epsilon_k * KELVIN_TO_ENERGY
            sig[i, i] = p.sigma
            lj[i, i] = 1 if p.lj else 0
        # applyMixingRule, Lorentz-Berthelot (forcefield.cpp:924-960)
        for i in range(n):
            for j in range(i + 1, n):
                if lj[i, i] and lj[j, j]:
                    m0 = math.sqrt(eps[i, i] * eps[j, j])
                    m1 = 0.5 * (sig[i, i] + sig[j, j])
                    eps[i, j] = eps[j, i] = m0
                    sig[i, j] = sig[j, i] = m1
                    lj[i, j] = lj[j, i] = 1
                else:
                    eps[i, j] = eps[j, i] = 0.0
                    sig[i, j] = sig[j, i] = 1.0
                    lj[i, j] = lj[j, i] = 0
        shift = np.zeros((n, n))
        if self.shifted:
            # preComputePotentialShift (forcefield.cpp:1038-1051) -> potentialEnergyAtFullCoupling(rc^2)
            for i in range(n):
                for j in range(n):
                    if not lj[i, j]:
                        continue
                    rc = self.cutoff_vdw(i, j)
                    temp = (rc * rc) / (sig[i, j] * sig[i, j])
                    rri3 = 1.0 / (temp * temp * temp)
                    shift[i, j] = 4.0 * eps[i, j] * (rri3 * (rri3 - 1.0))
        self.epsilon, self.sigma, self.shift, self.lj = eps, sig, shift, lj

    @property
    def n_types(self) -> int:
        return len(self.pseudo_atoms)

    def cutoff_vdw(self, i: int, j: int) -> float:
        """ForceField::cutOffVDW (forcefield.cpp:1016-1024)."""
        if self.pseudo_atoms[i].framework or self.pseudo_atoms[j].framework:
            return self.cutoff_framework_vdw
        return self.cutoff_molecule_vdw

    def index(self, name: str) -> int:
        for i, p in enumerate(self.pseudo_atoms):
            if p.name == name:
                return i
        raise KeyError(name)

    def use_sphere_kvectors(self):
        """Automatic-Ewald integer k-sphere: kx^2+ky^2+kz^2 <= max(kmax)^2 (forcefield.cpp:1434-1436)."""
        m = max(self.kmax)
        self.recip_int_cutoff_sq = m * m
        return self


# ---- C structs of the C-ABI (include/raspa_gpu.h) ----
class RgBox(ctypes.Structure):
    _fields_ = [("cell", ctypes.c_double * 9), ("triclinic", ctypes.c_int32)]


class RgForceField(ctypes.Structure):
    _fields_ = [
        ("n_types", ctypes.c_int32),
        ("epsilon", ctypes.POINTER(ctypes.c_double)),
        ("sigma", ctypes.POINTER(ctypes.c_double)),
        ("shift", ctypes.POINTER(ctypes.c_double)),
        ("lj", ctypes.POINTER(ctypes.c_int32)),
        ("cutoff_framework_vdw", ctypes.c_double),
        ("cutoff_molecule_vdw", ctypes.c_double),
        ("cutoff_coulomb", ctypes.c_double),
        ("ewald_alpha", ctypes.c_double),
        ("kmax_x", ctypes.c_int32), ("kmax_y", ctypes.c_int32), ("kmax_z", ctypes.c_int32),
        ("recip_int_cutoff_sq", ctypes.c_uint64),
        ("recip_cutoff_sq", ctypes.c_double),
        ("overlap_criteria", ctypes.c_double),
        ("use_charge", ctypes.c_int32),
        ("omit_inter", ctypes.c_int32),
    ]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def ff_struct(ff: ForceField, cls=RgForceField):
    """Build the C struct; the returned object keeps the table arrays alive."""
    eps = np.ascontiguousarray(ff.epsilon, dtype=np.float64)
    sig = np.ascontiguousarray(ff.sigma, dtype=np.float64)
    sh = np.ascontiguousarray(ff.shift, dtype=np.float64)
    lj = np.ascontiguousarray(ff.lj, dtype=np.int32)
    s = cls(ff.n_types, _dptr(eps), _dptr(sig), _dptr(sh), lj.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            ff.cutoff_framework_vdw, ff.cutoff_molecule_vdw, ff.cutoff_coulomb, ff.ewald_alpha,
            int(ff.kmax[0]), int(ff.kmax[1]), int(ff.kmax[2]), int(ff.recip_int_cutoff_sq), ff.recip_cutoff_sq,
            ff.overlap_criteria, 1 if ff.use_charge else 0, 1 if ff.omit_inter else 0)
    s._keep = (eps, sig, sh, lj)
    return s


def box_struct(cell, triclinic: bool | None = None, cls=RgBox):
    """cell: 3x3 with ROWS being the lattice vectors a, b, c (cell[i] = vector i)."""
    cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
    if triclinic is None:
        off = cell - np.diag(np.diag(cell))
        triclinic = bool(np.any(off != 0.0))
    b = cls()
    for i in range(9):
        b.cell[i] = float(cell.reshape(-1)[i])
    b.triclinic = 1 if triclinic else 0
    return b


def perpendicular_widths(cell) -> np.ndarray:
    """SimulationBox::perpendicularWidths (simulationbox.cpp:137-148); rows of cell are lattice vectors."""
    a, b, c = (np.asarray(v, dtype=np.float64) for v in np.asarray(cell).reshape(3, 3))
    c1, c2, c3 = np.cross(a, b), np.cross(b, c), np.cross(a, c)
    v = abs(float(np.dot(a, c2)))
    return np.array([v / math.sqrt(np.dot(c2, c2)), v / math.sqrt(np.dot(c3, c3)), v / math.sqrt(np.dot(c1, c1))])


def grid_points_for_spacing(cell, spacing: float) -> tuple[int, int, int]:
    """Grid size rule static_cast<size_t>(width/spacing + 0.5) (system_interpolation_grids.cpp:222-226)."""
    w = perpendicular_widths(cell)
    return tuple(int(x / spacing + 0.5) for x in w)

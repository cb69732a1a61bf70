"""Known-answer systems of the RASPA3 test suite, rebuilt from the published parameters.

* ``zeolite_forcefield`` restates ``ForceField::makeZeoliteForceField`` (src/raspakit/forcefield/forcefield.cpp:1777-1842):
  pseudo-atom charges and Lennard-Jones self parameters (epsilon in K, sigma in Angstrom), Lorentz-Berthelot mixing,
  one cutoff for all three cutoffs, shifted.
* ``itq29`` rebuilds ``Framework::makeITQ29`` (src/raspakit/framework.cpp:1561-1590): the four asymmetric-unit atoms
  expanded with space group Hall 517 (P m -3 m, symmorphic and primitive, 48 operations = every signed permutation of
  (x, y, z)), reduced to [0, 1) and de-duplicated within 0.1 Angstrom as ``CIFReader::expandDefinedAtomsToUnitCell``
  does (src/raspakit/cif_reader.cpp:589-631).
* ``co2_atoms`` / ``methane_atoms`` follow ``Component::makeCO2`` / ``makeMethane`` (src/raspakit/component.cpp:2290-2329).
"""

from __future__ import annotations

import itertools
import math

import numpy as np

from raspa3_b200.forcefield import ForceField, PseudoAtom, make_atoms

_ZEOLITE = [
    # name, framework, charge, epsilon_K, sigma
    ("-", False, 0.0, 1.0, 1.0),
    ("Si", True, 2.05, 22.0, 2.30),
    ("Al", True, 2.05, 22.0, 2.30),
    ("O", True, -1.025, 53.0, 3.30),
    ("Na+", False, 1.0, 15.0966, 2.65755),
    ("Cl-", False, -1.0, 142.562, 3.51932),
    ("CH4", False, 0.0, 158.5, 3.72),
    ("C_co2", False, 0.6512, 29.933, 2.745),
    ("O_co2", False, -0.3256, 85.671, 3.017),
    ("Ow", False, 0.0, 89.633, 3.097),
    ("Hw", False, 0.241, 0.0, 1.0),
    ("Lw", False, -0.241, 0.0, 1.0),
    ("probe-He", False, 0.0, 10.9, 2.64),
    ("probe-Ar", False, 0.0, 124.070, 3.38),
    ("probe-CH4", False, 0.0, 158.5, 3.72),
    ("probe-N2", False, 0.0, 91.5, 3.681),
]


def auto_ewald_alpha(cutoff_coulomb: float, precision: float = 1e-6) -> float:
    """The automatic Ewald alpha that System's constructor sets (ForceField::initializeEwaldParameters,
    src/raspakit/forcefield/forcefield.cpp:1415-1424): 0.26505830360350674 for a 12 Angstrom cutoff, where the
    force field's default is the rounded 0.265058."""
    eps = min(abs(precision), 0.5)
    tol = math.sqrt(abs(math.log(eps * cutoff_coulomb)))
    return math.sqrt(abs(math.log(eps * cutoff_coulomb * tol))) / cutoff_coulomb


def zeolite_forcefield(rc: float = 12.0, shifted: bool = True, use_charge: bool = True) -> ForceField:
    atoms = [PseudoAtom(n, fw, eps, sig, charge=q) for (n, fw, q, eps, sig) in _ZEOLITE]
    return ForceField(atoms, cutoff_framework_vdw=rc, cutoff_molecule_vdw=rc, cutoff_coulomb=rc, shifted=shifted,
                      use_charge=use_charge)


ITQ29_A = 11.8671
_ITQ29_ASYM = [
    # fractional position, pseudo-atom name, charge
    ((0.3683, 0.1847, 0.0), "Si", 2.05),
    ((0.5, 0.2179, 0.0), "O", -1.025),
    ((0.2939, 0.2939, 0.0), "O", -1.025),
    ((0.3429, 0.1098, 0.1098), "O", -1.025),
]


def _fract(v):
    s = v - np.rint(v)
    s = np.where(s < 0.0, s + 1.0, s)
    return np.where(s > 1.0, s - 1.0, s)


def _pm3m_images(p):
    out = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1.0, -1.0), repeat=3):
            out.append(np.array([signs[i] * p[perm[i]] for i in range(3)]))
    return out


def itq29(ff: ForceField, replicate=(1, 1, 1)):
    """ITQ-29 (LTA, P m -3 m): returns (cell rows, unit-cell atoms in Cartesian)."""
    a = ITQ29_A
    expanded = []
    for pos, name, q in _ITQ29_ASYM:
        for img in _pm3m_images(np.array(pos)):
            expanded.append((_fract(img), ff.index(name), q))
    keep = []
    for i, (fi, ti, qi) in enumerate(expanded):
        overlap = False
        for j in range(i + 1, len(expanded)):
            d = (fi - expanded[j][0]) * a
            d = d - np.rint(d / a) * a
            if float(d @ d) < 0.1 * 0.1:
                overlap = True
                break
        if not overlap:
            keep.append((fi, ti, qi))
    frac = np.array([k[0] for k in keep])
    types = np.array([k[1] for k in keep], dtype=np.uint16)
    charges = np.array([k[2] for k in keep])
    nx, ny, nz = replicate
    pos, tt, qq = [], [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                pos.append((frac + np.array([i, j, k])) * a)
                tt.append(types)
                qq.append(charges)
    cell = np.diag([a * nx, a * ny, a * nz])
    return cell, make_atoms(np.concatenate(pos), np.concatenate(tt), np.concatenate(qq))


# P n m a (space group 62, Hall "-P 2ac 2n", Hall number 292): the eight general positions of the standard setting
# (International Tables for Crystallography A, No. 62), as (rotation diagonal, translation).
_PNMA = [((1, 1, 1), (0.0, 0.0, 0.0)), ((-1, -1, 1), (0.5, 0.0, 0.5)), ((-1, 1, -1), (0.0, 0.5, 0.0)),
         ((1, -1, -1), (0.5, 0.5, 0.5)), ((-1, -1, -1), (0.0, 0.0, 0.0)), ((1, 1, -1), (0.5, 0.0, 0.5)),
         ((1, -1, 1), (0.0, 0.5, 0.0)), ((-1, 1, 1), (0.5, 0.5, 0.5))]


def mfi(ff: ForceField, replicate=(1, 1, 1)):
    """MFI (Framework::makeMFI, src/raspakit/framework.cpp:1591-1660): the asymmetric unit of tests/golden/
    mfi_framework.json (generated from that source by tests/golden/make_mfi_fixture.py) expanded with P n m a,
    reduced to [0, 1) and de-duplicated within 0.1 Angstrom as CIFReader::expandDefinedAtomsToUnitCell does
    (cif_reader.cpp:589-631). Returns (cell rows, unit-cell or replicated atoms in Cartesian)."""
    import json
    import os

    d = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mfi_framework.json")))
    assert d["hall_number"] == 292
    L = np.asarray(d["cell_lengths"])
    expanded = []
    for x, y, z, q, name in d["asymmetric_atoms"]:
        p = np.array([x, y, z])
        for rot, tr in _PNMA:
            expanded.append((_fract(np.asarray(rot) * p + np.asarray(tr)), ff.index(name), q))
    keep = []
    for i, (fi, ti, qi) in enumerate(expanded):
        dup = False
        for j in range(i + 1, len(expanded)):
            dd = (fi - expanded[j][0]) * L
            dd = dd - np.rint(dd / L) * L
            if float(dd @ dd) < 0.1 * 0.1:
                dup = True
                break
        if not dup:
            keep.append((fi, ti, qi))
    frac = np.array([k[0] for k in keep])
    types = np.array([k[1] for k in keep], dtype=np.uint16)
    charges = np.array([k[2] for k in keep])
    nx, ny, nz = replicate
    pos, tt, qq = [], [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                pos.append((frac + np.array([i, j, k])) * L)
                tt.append(types)
                qq.append(charges)
    cell = np.diag(L * np.array(replicate, dtype=np.float64))
    return cell, make_atoms(np.concatenate(pos), np.concatenate(tt), np.concatenate(qq))


def co2_atoms(ff: ForceField, centers, molecule_ids, bond=1.149, axis=(0.0, 0.0, 1.0), charges=True):
    """Rigid CO2 (O, C, O order of Component::makeCO2) centred at each point along `axis`."""
    qO, qC = (-0.3256, 0.6512) if charges else (0.0, 0.0)
    tO, tC = ff.index("O_co2"), ff.index("C_co2")
    ax = np.asarray(axis, dtype=np.float64)
    pos, types, qs, mids = [], [], [], []
    for c, m in zip(np.asarray(centers, dtype=np.float64).reshape(-1, 3), molecule_ids):
        pos += [c + bond * ax, c, c - bond * ax]
        types += [tO, tC, tO]
        qs += [qO, qC, qO]
        mids += [m, m, m]
    return make_atoms(np.array(pos), np.array(types, dtype=np.uint16), np.array(qs), molecule_ids=np.array(mids))


def methane_atoms(ff: ForceField, positions, molecule_ids):
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    return make_atoms(p, ff.index("CH4"), 0.0, molecule_ids=np.asarray(molecule_ids))

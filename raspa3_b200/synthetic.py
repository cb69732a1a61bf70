"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

No public structure files are used: frameworks are generated, deterministically from a seed, with the sizes, atom
counts and parameter values of each configuration.

Framework placement algorithm (``synthetic_framework``), orthorhombic cell:
  1. T atoms: uniform random fractional positions (numpy PCG64 from the seed), accepted when the minimum-image
     distance to every T atom already placed is at least ``t_sep`` (3.0 Angstrom, room for the bonded O atoms).
  2. O atoms: for each T atom in order, two O atoms at ``bond`` (1.6 Angstrom) along uniform random directions,
     accepted when the minimum-image distance to every other atom placed so far is at least ``min_sep``
     (1.5 Angstrom). Every T-O bonded pair is therefore at exactly 1.6 Angstrom and every other pair at >= 1.5.
  The unit cell holds n_T T atoms and 2 n_T O atoms (96 + 192 for the 20.0 x 19.9 x 13.4 A cell and its replicas).
"""

from __future__ import annotations

import math

import numpy as np

from .forcefield import ForceField, PseudoAtom, grid_points_for_spacing, make_atoms

SYNTHETIC_CELL = (20.0, 19.9, 13.4)
GRID_SPACING = 0.15


def synthetic_forcefield(rc: float = 12.0, charges: bool = True, alpha: float = 0.265, kmax: int = 8,
                         sphere: bool = True) -> ForceField:
    """Pseudo-atoms of the benchmark configurations (epsilon in K, sigma in Angstrom, charge in e).

    T carries no Lennard-Jones term; N_com is the massless charge site of 3-site N2. Ewald: alpha and kmax as given,
    integer k-sphere kx^2+ky^2+kz^2 <= kmax^2 when `sphere` (the automatic-Ewald semantic), else the full half-box.
    """
    q = (lambda v: v) if charges else (lambda v: 0.0)
    atoms = [
        PseudoAtom("T", True, 0.0, 1.0, charge=q(2.05), lj=False),
        PseudoAtom("O", True, 89.6, 3.0, charge=q(-1.025)),
        PseudoAtom("CH4", False, 158.5, 3.72, charge=0.0),
        PseudoAtom("C_co2", False, 27.0, 2.80, charge=q(0.70)),
        PseudoAtom("O_co2", False, 79.0, 3.05, charge=q(-0.35)),
        PseudoAtom("N_n2", False, 36.0, 3.31, charge=q(-0.482)),
        PseudoAtom("N_com", False, 0.0, 1.0, charge=q(0.964), lj=False),
        PseudoAtom("CH3", False, 98.0, 3.75, charge=0.0),
        PseudoAtom("CH2", False, 46.0, 3.95, charge=0.0),
    ]
    ff = ForceField(atoms, cutoff_framework_vdw=rc, cutoff_molecule_vdw=rc, cutoff_coulomb=rc, shifted=True,
                    ewald_alpha=alpha, kmax=(kmax, kmax, kmax), use_charge=charges)
    if sphere:
        ff.use_sphere_kvectors()
    return ff


def _min_image(d, L):
    return d - L * np.rint(d / L)


def synthetic_framework(ff: ForceField, lengths=SYNTHETIC_CELL, n_t: int = 96, seed: int = 42, min_sep: float = 1.5,
                        t_sep: float = 3.0, bond: float = 1.6, max_tries: int = 200000):
    """Returns (cell rows 3x3, unit-cell atom records). Charges come from the force field's pseudo-atoms."""
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths, dtype=np.float64)
    t_pos = np.zeros((0, 3))
    tries = 0
    while len(t_pos) < n_t:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("synthetic_framework: could not place T atoms")
        p = rng.random(3) * L
        if len(t_pos):
            d = _min_image(t_pos - p, L)
            if np.min(np.einsum("ij,ij->i", d, d)) < t_sep * t_sep:
                continue
        t_pos = np.vstack([t_pos, p])
    all_pos = t_pos.copy()
    o_pos = []
    for t in range(n_t):
        placed = 0
        while placed < 2:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("synthetic_framework: could not place O atoms")
            v = rng.normal(size=3)
            v /= np.linalg.norm(v)
            p = np.mod(t_pos[t] + bond * v, L)
            d = _min_image(all_pos - p, L)
            r2 = np.einsum("ij,ij->i", d, d)
            r2[t] = np.inf  # its own T atom sits at the bond length
            if np.min(r2) < min_sep * min_sep:
                continue
            all_pos = np.vstack([all_pos, p])
            o_pos.append(p)
            placed += 1
    o_pos = np.array(o_pos)
    tT, tO = ff.index("T"), ff.index("O")
    qT, qO = ff.pseudo_atoms[tT].charge, ff.pseudo_atoms[tO].charge
    pos = np.vstack([t_pos, o_pos])
    types = np.array([tT] * n_t + [tO] * (2 * n_t), dtype=np.uint16)
    charges = np.array([qT] * n_t + [qO] * (2 * n_t))
    cell = np.diag(L)
    return cell, make_atoms(pos, types, charges)


def replicate(cell, atoms, reps):
    """Framework::makeSuperCell order (framework.cpp:1085-1102): i outer, k inner, atoms innermost."""
    cell = np.asarray(cell, dtype=np.float64)
    out = []
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                a = atoms.copy()
                shift = i * cell[0] + j * cell[1] + k * cell[2]
                a["x"] += shift[0]
                a["y"] += shift[1]
                a["z"] += shift[2]
                out.append(a)
    big = cell * np.asarray(reps, dtype=np.float64)[:, None]
    return big, np.concatenate(out)


def spacing_grid_dims(cell=None):
    """133 x 133 x 89 for the 20.0 x 19.9 x 13.4 Angstrom cell at 0.15 Angstrom spacing."""
    return grid_points_for_spacing(np.diag(SYNTHETIC_CELL) if cell is None else cell, GRID_SPACING)


def batched_frameworks(ff: ForceField, n_systems: int = 64, seed: int = 1234, density: float = 288 / 5333.2,
                       lmin: float = 12.0, lmax: float = 40.0, nmin: int = 96, nmax: int = 1536):
    """The batched-alkane frameworks: cells with lengths uniform in [12, 40] Angstrom and 96-1536 atoms (count set by the
    density of the 20.0 x 19.9 x 13.4 A cell, clipped to the range, rounded to a multiple of 3 so that T:O = 1:2)."""
    rng = np.random.default_rng(seed)
    systems = []
    for s in range(n_systems):
        L = rng.uniform(lmin, lmax, size=3)
        n = int(np.clip(round(density * float(np.prod(L))), nmin, nmax))
        n_t = max(1, n // 3)
        # dense small cells need a smaller T exclusion; keep the 1.5 Angstrom global minimum
        vol_per_t = float(np.prod(L)) / n_t
        t_sep = min(3.0, 0.8 * vol_per_t ** (1.0 / 3.0))
        cell, atoms = synthetic_framework(ff, tuple(L), n_t=n_t, seed=int(rng.integers(1 << 31)), t_sep=t_sep)
        systems.append((cell, atoms))
    return systems


def random_rotation(rng) -> np.ndarray:
    """Uniform random rotation matrix (from a uniform unit quaternion)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def rigid_molecule(ff: ForceField, names, offsets, center, rotation, molecule_id, lam: float = 1.0, group: int = 0,
                   fractional: bool = False):
    """Atoms of a rigid molecule: body-frame offsets rotated and translated to `center`."""
    from .forcefield import lambda_scaling

    offsets = np.asarray(offsets, dtype=np.float64)
    pos = np.asarray(center, dtype=np.float64)[None, :] + offsets @ np.asarray(rotation).T
    types = np.array([ff.index(n) for n in names], dtype=np.uint16)
    charges = np.array([ff.pseudo_atoms[t].charge for t in types])
    svdw, scoul = lambda_scaling(lam) if lam != 1.0 else (1.0, 1.0)
    n = len(names)
    return make_atoms(pos, types, charges, molecule_ids=np.full(n, molecule_id), scaling_vdw=svdw,
                      scaling_coulomb=scoul, group_ids=np.full(n, group), fractional=np.full(n, 1 if fractional else 0))


CO2_NAMES = ("O_co2", "C_co2", "O_co2")
CO2_OFFSETS = ((0.0, 0.0, 1.16), (0.0, 0.0, 0.0), (0.0, 0.0, -1.16))
N2_NAMES = ("N_n2", "N_com", "N_n2")
N2_OFFSETS = ((0.0, 0.0, 0.55), (0.0, 0.0, 0.0), (0.0, 0.0, -0.55))


def random_molecules(ff: ForceField, cell, n: int, names=CO2_NAMES, offsets=CO2_OFFSETS, seed: int = 0,
                     first_id: int = 0):
    """n rigid molecules at uniform random positions and orientations (no overlap test)."""
    rng = np.random.default_rng(seed)
    cell = np.asarray(cell, dtype=np.float64)
    mols = [rigid_molecule(ff, names, offsets, rng.random(3) @ cell, random_rotation(rng), first_id + i)
            for i in range(n)]
    return np.concatenate(mols) if mols else make_atoms(np.zeros((0, 3)), np.zeros(0, np.uint16), np.zeros(0))

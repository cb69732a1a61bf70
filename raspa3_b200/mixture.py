"""The large two-component system: CO2 and N2 in a synthetic charged framework replicated 4 x 4 x 4.

The framework is the synthetic charged generator (96 T + 192 O per cell, T +2.05 e, O -1.025 e) on a cell 1.5 times
the 20.0 x 19.9 x 13.4 A cell's lengths (30.0 x 29.85 x 20.1 A), replicated 4 x 4 x 4: 18,432 atoms, holding 2,000 rigid CO2
and 2,000 rigid 3-site N2 (N-N 1.10 A, N 36 K / 3.31 A / -0.482 e, massless centre +0.964 e); Ewald alpha = 0.265 per
Angstrom and kmax 12 given explicitly, so every k of the half-box is used, as the reference does for explicit Ewald
parameters (forcefield.cpp:388-418; 8,124 k-vectors; the integer sphere belongs to the automatic setting). Framework
energies come from the unit-cell grids (C_co2, O_co2, N_n2 and N_com Lennard-Jones -- every adsorbate type has one,
N_com's being zero -- and the unit-charge real-space Ewald grid, 0.15 A spacing). The larger cell is what makes room for
4,000 molecules: in the 20.0 x 19.9 x 13.4 A cell with randomly placed atoms only 0.7 % of the volume is farther than
2.6 A from an atom, too little for 62.5 molecules per cell; at 1.5 times the lengths it is 44 %.
"""

from __future__ import annotations

import numpy as np

from .forcefield import ENERGY_TO_KELVIN, grid_points_for_spacing, make_atoms
from .gcmc import co2_component, n2_component
from .synthetic import random_rotation, replicate, synthetic_forcefield, synthetic_framework


def random_mixture(cell, framework, components, counts, seed: int = 5, min_fw: float = 2.6, min_mol: float = 2.8,
                   max_tries: int = 2_000_000):
    """Random non-overlapping rigid molecules: counts[c] of components[c] with no atom closer than min_fw to a
    framework atom or min_mol to another molecule's atom (periodic orthorhombic box). Every molecule is whole: its
    atoms are the rigid offsets about a point in the box, not wrapped one by one. Returns (xyz[n, na, 3], comp[n])."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    L = np.diag(np.asarray(cell))
    fw = np.stack([framework["x"], framework["y"], framework["z"]], 1) % L
    fw_tree = cKDTree(fw, boxsize=L)
    order = np.concatenate([np.full(n, c) for c, n in enumerate(counts)])
    rng.shuffle(order)
    placed, comps = [], []
    grid_size = 4.0
    cells: dict = {}

    def near(p):
        k = tuple((p // grid_size).astype(int))
        dims = np.maximum(1, (L // grid_size).astype(int))
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((k[0] + dx) % dims[0], (k[1] + dy) % dims[1], (k[2] + dz) % dims[2])
                    for q in cells.get(kk, ()):
                        d = q - p
                        d -= np.rint(d / L) * L
                        if d @ d < min_mol * min_mol:
                            return True
        return False

    tries = 0
    for c in order:
        comp = components[c]
        while True:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("random_mixture: could not place the molecules")
            # the molecule stays whole (atoms may lie outside the box); distances use the wrapped copy
            x = comp.offsets @ random_rotation(rng).T + rng.random(3) * L
            xw = x % L
            if fw_tree.query(xw, k=1)[0].min() < min_fw:
                continue
            if any(near(a) for a in xw):
                continue
            break
        dims = np.maximum(1, (L // grid_size).astype(int))
        for a in xw:
            k = tuple(((a // grid_size).astype(int)) % dims)
            cells.setdefault(k, []).append(a)
        placed.append(x)
        comps.append(c)
    return np.array(placed), np.array(comps, dtype=np.int32)


def molecules_as_atoms(ff, components, xyz, comp):
    """rg_atom records of the molecules (molecule id = index)."""
    na = xyz.shape[1]
    types = np.concatenate([components[c].types(ff) for c in comp]).astype(np.uint16)
    charges = np.concatenate([components[c].charges(ff) for c in comp])
    ids = np.repeat(np.arange(len(comp), dtype=np.uint32), na)
    return make_atoms(xyz.reshape(-1, 3), types, charges, molecule_ids=ids)


def total_energy(system, ewald, ff, components, xyz, comp):
    """Total energy of a configuration on the device (internal units): framework (grids) + molecule-molecule pairs
    (each counted once) + Ewald Fourier, self and exclusion terms."""
    atoms = molecules_as_atoms(ff, components, xyz, comp)
    system.set_molecules(atoms)
    na = xyz.shape[1]
    per = 4096 // na  # rg_cbmc_external_energies takes at most 4096 trial atoms per call
    fw = mm = 0.0
    for b in range(0, len(comp), per):
        for r in system.external_energies(atoms[b * na:(b + per) * na], na):
            fw += r.framework_vdw + r.framework_charge
            mm += 0.5 * (r.molecule_vdw + r.molecule_charge)
    e = ewald.full(atoms, np.full(len(comp), na, dtype=np.int32))
    return fw + mm + e["ewald_fourier"] + e["ewald_self"] + e["ewald_exclusion"]


MIXTURE_CELL = (30.0, 29.85, 20.1)


def large_mixture(ctx, torch, reps=(4, 4, 4), counts=(2000, 2000), kmax: int = 12, seed: int = 5, dims=None,
            lengths=MIXTURE_CELL, spacing: float = 0.15):
    """Builds the large mixture system: returns a dict with the force field, cells, framework, grids (device buffers
    kept alive), System, Ewald, components and the starting configuration."""
    from . import native

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=kmax, sphere=False)
    ucell, ufw = synthetic_framework(ff, lengths, n_t=96, seed=42)
    scell, sfw = replicate(ucell, ufw, reps)
    dims = dims or grid_points_for_spacing(ucell, spacing)
    system = native.System(ctx, ff, scell, sfw)
    bufs, grid_types = [], []
    for name in ("C_co2", "O_co2", "N_n2", "N_com"):
        idx = ff.index(name)
        buf = torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
        ctx.grid_build(0, ff, ucell, ufw, idx, 12.0, dims, native.PRECISION_FP32C, out_device=buf.data_ptr(),
                       host=False)
        system.set_grid(idx, ucell, dims, buf.data_ptr(), on_device=True)
        bufs.append(buf)
        grid_types.append(idx)
    buf = torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
    ctx.grid_build(1, ff, ucell, ufw, 0, 12.0, dims, native.PRECISION_FP32C, out_device=buf.data_ptr(), host=False)
    system.set_grid(ff.n_types, ucell, dims, buf.data_ptr(), on_device=True)
    bufs.append(buf)
    grid_types.append(ff.n_types)
    ewald = native.Ewald(ctx, ff, scell)
    ewald.set_framework(sfw)
    components = [co2_component(), n2_component()]
    xyz, comp = random_mixture(scell, sfw, components, counts, seed=seed)
    return {"ff": ff, "unit_cell": ucell, "unit_framework": ufw, "cell": scell, "framework": sfw, "grids": bufs,
            "grid_types": grid_types, "system": system, "ewald": ewald, "components": components, "xyz": xyz, "comp": comp, "dims": dims}


def kelvin(e: float) -> float:
    return e * ENERGY_TO_KELVIN

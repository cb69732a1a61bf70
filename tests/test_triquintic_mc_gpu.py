"""Triquintic grids inside the device-resident Monte Carlo drivers: the GCMC chains (rg_gcmc), the large-mixture kernel
(rg_mixture) and the learned proposal's grid-sampled targets (rg_proposal_sample_targets) interpolate a system whose
grids hold the 27 triquintic values per point (InterpolationEnergyGrid::interpolate, triquintic branch,
interpolation_energy_grid.cpp:4119-4178). Checked against FP64 recomputations whose grid part is the oracle's
triquintic interpolant."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, n2_component
from raspa3_b200.mixture import random_mixture, total_energy
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu
BETA = beta_of(300.0)


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def triquintic_system(ctx, types, charges=True, kmax=8, dims=(33, 33, 23)):
    """The charged synthetic framework in its 2x2x3 box with triquintic grids of the given pseudo-atom names and the
    unit-charge Ewald grid."""
    ff = synthetic_forcefield(charges=charges, alpha=0.265, kmax=kmax)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    sysg = native.System(ctx, ff, scell, sfw)
    sysg.set_interpolation_scheme(native.SCHEME_TRIQUINTIC)
    grids = [None] * (ff.n_types + 1)
    specs = [(ff.index(t), native.GRID_LENNARD_JONES) for t in types]
    if charges:
        specs.append((ff.n_types, native.GRID_EWALD_REAL))
    for idx, gt in specs:
        out, _ = ctx.grid_build_triquintic(gt, ff, ucell, ufw, idx if gt == native.GRID_LENNARD_JONES else 0, 12.0,
                                           dims)
        grids[idx] = out
        sysg.set_grid(idx, ucell, dims, out)
    ew = native.Ewald(ctx, ff, scell) if charges else None
    if ew is not None:
        ew.set_framework(sfw)
    return dict(ff=ff, ucell=ucell, scell=scell, sfw=sfw, dims=dims, grids=grids, sys=sysg, ew=ew)


def grid_energy(oracle, s, types, charges, xyz):
    """Framework energy of atoms from the triquintic grids: the type's VDW grid plus charge x unit-charge Ewald grid."""
    e = 0.0
    ff = s["ff"]
    for t, q, r in zip(types, charges, xyz):
        if s["grids"][t] is not None:
            e += oracle.interpolate_triquintic(s["grids"][t], s["dims"], s["ucell"], r)[0]
            if ff.use_charge and q != 0.0:
                e += q * oracle.interpolate_triquintic(s["grids"][ff.n_types], s["dims"], s["ucell"], r)[0]
    return e


def test_gcmc_with_triquintic_grids_keeps_its_energy(ctx, oracle):
    s = triquintic_system(ctx, ["C_co2", "O_co2"])
    ff, comp = s["ff"], co2_component()
    g = native.Gcmc(s["sys"], s["ew"], comp, BETA, fugacity_of(1e5), n_chains=64, seed=17)
    g.run(3000, record=True)
    res = g.results()
    assert np.mean([r["n_molecules"] for r in res]) > 1
    s_fw = oracle.ewald_rigid(ff, s["scell"], s["sfw"])
    for ch in range(3):
        xyz = g.positions(ch)
        n_mol = len(xyz) // comp.n_atoms
        types = np.tile(comp.types(ff), n_mol)
        q = np.tile(comp.charges(ff), n_mol)
        atoms = make_atoms(xyz, types.astype(np.uint16), q, molecule_ids=np.repeat(np.arange(n_mol), comp.n_atoms))
        e = grid_energy(oracle, s, types, q, xyz)
        for m in range(n_mol):
            mol = atoms[m * comp.n_atoms:(m + 1) * comp.n_atoms]
            ok, em = oracle.cbmc_intermolecular(ff, s["scell"], atoms[(m + 1) * comp.n_atoms:], mol,
                                                ff.cutoff_molecule_vdw, ff.cutoff_coulomb)
            e += em["molecule_molecule_vdw"] + em["molecule_molecule_charge"]
        if n_mol:
            ee, _ = oracle.ewald_fourier_energy(ff, s["scell"], atoms, [comp.n_atoms] * n_mol, s_rigid=s_fw)
            e += ee["ewald_fourier"] + ee["ewald_self"] + ee["ewald_exclusion"]
        assert abs(e - res[ch]["energy"]) <= 1e-6 * max(1.0, abs(e)), (ch, e, res[ch]["energy"])


def test_mixture_with_triquintic_grids_keeps_its_energy(ctx):
    s = triquintic_system(ctx, ["C_co2", "O_co2", "N_n2"])
    ff, comps = s["ff"], [co2_component(), n2_component()]
    xyz, comp = random_mixture(s["scell"], s["sfw"], comps, (8, 8), seed=21)
    e0 = total_energy(s["sys"], s["ew"], ff, comps, xyz, comp)
    mx = native.Mixture(s["sys"], s["ew"], comps, BETA, [fugacity_of(1e6), fugacity_of(1e6)], xyz, comp,
                        max_molecules=128, seed=5, n_blocks=37)
    mx.set_state(e0, s["ew"].structure_factors(0))
    mx.run(1500)
    r = mx.results()
    assert r["status"] == 0 and sum(r["accepted"]) > 0
    xyz1, comp1 = mx.positions()
    e = total_energy(s["sys"], s["ew"], ff, comps, xyz1, comp1)
    assert abs(r["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (r["energy"], e)
    mx.close()


def test_proposal_targets_from_triquintic_grids(ctx, oracle):
    import torch

    s = triquintic_system(ctx, ["C_co2"])
    ff = s["ff"]
    t_min = -15.0
    pa = ff.index("C_co2")
    charge = float(co2_component().charges(ff)[co2_component().starting_bead])
    n = 4096
    sd = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    td = torch.empty(n, dtype=torch.float32, device="cuda")
    native.sample_targets(s["sys"], pa, charge, BETA, t_min, s["ucell"], n, 7, sd.data_ptr(), td.data_ptr())
    torch.cuda.synchronize()
    su, tu = sd.cpu().numpy().astype(np.float64), td.cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(3)
    for i in rng.choice(n, 200, replace=False):
        # the device samples s in FP64 and stores it in FP32: recompute at the stored point, compare loosely where the
        # energy is steep (a float32 rounding of s moves the point by ~1e-6 A)
        r = su[i] @ s["ucell"]
        e = grid_energy(oracle, s, [pa], [charge], [r])
        ref = max(-BETA * e, t_min)
        assert abs(tu[i] - ref) <= 1e-4 * max(1.0, abs(ref)) + 1e-3, (i, tu[i], ref)

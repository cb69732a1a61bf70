"""(b) CBMC trial energies on the GPU through the C-ABI vs the FP64 oracle and the reference goldens."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ENERGY_TO_KELVIN, make_atoms
from raspa3_b200.synthetic import (CO2_NAMES, CO2_OFFSETS, random_molecules, random_rotation, replicate,
                                   rigid_molecule, synthetic_forcefield, synthetic_framework)
from reference_systems import ITQ29_A, itq29, methane_atoms, zeolite_forcefield

pytestmark = pytest.mark.gpu

FIELDS = ("framework_vdw", "framework_charge", "molecule_vdw", "molecule_charge")
ORACLE = {"framework_vdw": "framework_molecule_vdw", "framework_charge": "framework_molecule_charge",
          "molecule_vdw": "molecule_molecule_vdw", "molecule_charge": "molecule_molecule_charge"}


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def test_golden_methane_itq29(ctx):
    """tests/raspakit-tests/cbmc_interactions.cpp:27-90 through rg_cbmc_external_energies (pair-loop branch)."""
    ff = zeolite_forcefield(12.0, True, use_charge=False)
    cell, fw = itq29(ff)
    sysg = native.System(ctx, ff, cell, fw)
    a = ITQ29_A
    one = methane_atoms(ff, [(0.5 * a, 0.5 * a, 0.5 * a)], [0])
    sysg.set_molecules(one[:0])
    (e,) = sysg.external_energies(one, 1)
    assert abs(e.framework_vdw * ENERGY_TO_KELVIN - (-337.77056357)) < 1e-6
    two = methane_atoms(ff, [(0.5 * a, 0.5 * a, 0.5 * a), (0.6 * a, 0.7 * a, 0.65 * a)], [0, 1])
    sysg.set_molecules(two)
    e0, e1 = sysg.external_energies(two, 1)
    assert abs((e0.framework_vdw + e1.framework_vdw) * ENERGY_TO_KELVIN - (-1599.10322574)) < 1e-6
    assert abs(e0.molecule_vdw * ENERGY_TO_KELVIN - 2352.42793591) < 1e-6
    assert abs(e1.molecule_vdw * ENERGY_TO_KELVIN - 2352.42793591) < 1e-6


@pytest.fixture(scope="module")
def config2(ctx):
    """Configuration-2 system: charged framework in a 2x2x3 simulation box, FP64 grids on a 0.5 A mesh, 30 CO2."""
    ff = synthetic_forcefield(charges=True)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (41, 41, 28)
    grids = {}
    for idx, gt in ((ff.index("C_co2"), 0), (ff.index("O_co2"), 0), (ff.n_types, 1)):
        probe = idx if gt == 0 else 0
        out, _ = ctx.grid_build(gt, ff, ucell, ufw, probe, 12.0, dims, native.PRECISION_FP64)
        grids[idx] = out
    ads = random_molecules(ff, scell, 30, seed=8)
    sysg = native.System(ctx, ff, scell, sfw)
    for idx, g in grids.items():
        sysg.set_grid(idx, ucell, dims, g)
    sysg.set_molecules(ads)
    oracle_grids = [None] * (ff.n_types + 1)
    for idx, g in grids.items():
        oracle_grids[idx] = g
    return dict(ff=ff, ucell=ucell, scell=scell, sfw=sfw, dims=dims, grids=oracle_grids, ads=ads, sys=sysg)


def oracle_trial(oracle, c, trial, skip=-1, skip_background=-1, grids=True):
    ff = c["ff"]
    ok1, e1 = oracle.cbmc_framework_molecule(ff, c["scell"], c["sfw"], trial, ff.cutoff_framework_vdw,
                                             ff.cutoff_coulomb, grids=c["grids"] if grids else None,
                                             grid_dims=c["dims"], grid_cell=c["ucell"], skip=skip)
    ok2, e2 = oracle.cbmc_intermolecular(ff, c["scell"], c["ads"], trial, ff.cutoff_molecule_vdw, ff.cutoff_coulomb,
                                         skip=skip, skip_background=skip_background)
    e = {k: e1[ORACLE[k]] + e2[ORACLE[k]] for k in FIELDS}
    e["dudlambda_vdw"] = np.add(e1["dudlambda_vdw"], e2["dudlambda_vdw"])
    e["dudlambda_charge"] = np.add(e1["dudlambda_charge"], e2["dudlambda_charge"])
    return ok1 and ok2, e


def check(gpu, ok, ref):
    assert bool(gpu.overlap) == (not ok)
    if not ok:
        return
    for k in FIELDS:
        assert abs(getattr(gpu, k) - ref[k]) <= 1e-9 * max(1.0, abs(ref[k])), (k, getattr(gpu, k), ref[k])


def test_first_bead_trials_grid_branch(config2, oracle):
    c = config2
    ff = c["ff"]
    rng = np.random.default_rng(21)
    pos = rng.random((10, 3)) @ c["scell"]
    trials = make_atoms(pos, ff.index("C_co2"), 0.70, molecule_ids=np.full(10, 30))
    got = c["sys"].external_energies(trials, 1)
    n_ok = 0
    for t in range(10):
        ok, ref = oracle_trial(oracle, c, trials[t:t + 1])
        check(got[t], ok, ref)
        n_ok += ok
    assert n_ok >= 1


def test_orientation_trials_with_skip(config2, oracle):
    """Chain-growth trial sets (three CO2 atoms around a fixed first bead, first bead skipped)."""
    c = config2
    ff = c["ff"]
    rng = np.random.default_rng(5)
    center = rng.random(3) @ c["scell"]
    sets = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, center, random_rotation(rng), 30) for _ in range(10)]
    trials = np.concatenate(sets)
    got = c["sys"].external_energies(trials, 3, skip=1)
    for t in range(10):
        ok, ref = oracle_trial(oracle, c, sets[t], skip=1)
        check(got[t], ok, ref)


def test_pair_loop_branch_fractional_and_groups(config2, oracle):
    """A fractional CFCMC molecule (no grid branch): framework pair loop over 3456 atoms, lambda 0.6, group 1."""
    c = config2
    ff = c["ff"]
    rng = np.random.default_rng(6)
    sets = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 31, lam=0.6,
                           group=1, fractional=True) for _ in range(6)]
    trials = np.concatenate(sets)
    got = c["sys"].external_energies(trials, 3)
    for t in range(6):
        ok, ref = oracle_trial(oracle, c, sets[t])
        check(got[t], ok, ref)
        if ok:
            np.testing.assert_allclose(got[t].dudlambda_vdw[:], ref["dudlambda_vdw"], rtol=1e-9, atol=1e-9)
            np.testing.assert_allclose(got[t].dudlambda_charge[:], ref["dudlambda_charge"], rtol=1e-9, atol=1e-9)


def test_skip_background_molecule(config2, oracle):
    c = config2
    ff = c["ff"]
    old = c["ads"][6:9]  # molecule 2, retraced: its own interactions are skipped by moleculeId
    trial = old.copy()
    got = c["sys"].external_energies(trial, 3, skip_background=2)
    ok, ref = oracle_trial(oracle, c, trial, skip_background=2)
    check(got[0], ok, ref)


def test_fp32c_trial_energies(config2, oracle):
    """RG_PRECISION_FP32C: FP32 pair terms from the FP64 minimum-image displacement, TwoSum-compensated FP32 sums.
    Bound: a trial's energy (the sum of its framework / molecule, VDW / charge parts) agrees with the FP64 oracle within
    1e-6 of the sum of the parts' magnitudes, and each VDW part within 1e-5 of itself. A charge part alone can be
    further off relative to itself where +2.05 / -1.025 e terms cancel (measured up to 6e-4 for the framework charge of
    a fractional molecule, whose pair loop runs over the charged framework atoms)."""
    c = config2
    ff = c["ff"]
    rng = np.random.default_rng(23)
    first = make_atoms(rng.random((20, 3)) @ c["scell"], ff.index("C_co2"), 0.70, molecule_ids=np.full(20, 30))
    orient = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 30)
              for _ in range(10)]
    frac = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 31, lam=0.6,
                           group=1, fractional=True) for _ in range(6)]
    c["sys"].set_precision(native.PRECISION_FP32C)
    try:
        cases = [(c["sys"].external_energies(first, 1), [first[t:t + 1] for t in range(20)], -1),
                 (c["sys"].external_energies(np.concatenate(orient), 3, skip=1), orient, 1),
                 (c["sys"].external_energies(np.concatenate(frac), 3), frac, -1)]
    finally:
        c["sys"].set_precision(native.PRECISION_FP64)
    n_ok = 0
    for got, sets, skip in cases:
        for g, s in zip(got, sets):
            ok, ref = oracle_trial(oracle, c, s, skip=skip)
            assert bool(g.overlap) == (not ok)
            if not ok:
                continue
            n_ok += 1
            scale = sum(abs(ref[k]) for k in FIELDS)
            total = sum(getattr(g, k) for k in FIELDS)
            assert abs(total - sum(ref[k] for k in FIELDS)) <= 1e-6 * max(1.0, scale), (total, ref)
            for k in ("framework_vdw", "molecule_vdw"):
                assert abs(getattr(g, k) - ref[k]) <= 1e-5 * max(1.0, abs(ref[k])), (k, getattr(g, k), ref[k])
    assert n_ok >= 10

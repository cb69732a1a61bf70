"""(b) CBMC trial energies on the GPU through the C-ABI vs the FP64 oracle and the reference goldens."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ENERGY_TO_KELVIN, make_atoms
from raspa3_b200.synthetic import (CO2_NAMES, CO2_OFFSETS, random_molecules, random_rotation, replicate,
                                   rigid_molecule, synthetic_forcefield, synthetic_framework)
from reference_systems import ITQ29_A, itq29, methane_atoms, zeolite_forcefield
from test_oracle_golden import STATIC_CO2_ITQ29, STATIC_CO2_MFI, static_co2_itq29_system, static_co2_mfi_system

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


@pytest.mark.parametrize("precision", [native.PRECISION_FP64, native.PRECISION_FP32C])
def test_golden_two_co2_itq29_charged(ctx, precision):
    """tests/raspakit-tests/static_energy.cpp:21-46 through rg_cbmc_external_energies: the real-space Ewald Coulomb
    pair (potentialCoulomb<0>) against the charged ITQ-29 framework and between the two CO2, and the Lennard-Jones
    terms, to 1e-6 K in FP64; in FP32C (Lennard-Jones pairs in FP32) each term within 1e-6 of itself."""
    ff, cell, fw, atoms = static_co2_itq29_system()
    sysg = native.System(ctx, ff, cell, fw)
    sysg.set_precision(precision)
    sysg.set_molecules(atoms)
    trials = sysg.external_energies(atoms, 1)  # one trial per atom: framework terms, and molecule terms vs the other CO2
    fw_vdw = sum(t.framework_vdw for t in trials)
    fw_q = sum(t.framework_charge for t in trials)
    mm_vdw = sum(t.molecule_vdw for t in trials[:3])
    mm_q = sum(t.molecule_charge for t in trials[:3])
    got = np.array([fw_vdw, fw_q, mm_vdw, mm_q]) * ENERGY_TO_KELVIN
    ref = np.array(STATIC_CO2_ITQ29)
    if precision == native.PRECISION_FP64:
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6)
    else:
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=0)
    sysg.close()


def test_golden_two_co2_mfi_charged(ctx):
    """tests/raspakit-tests/static_energy.cpp:48-74 (2 CO2 in MFI 2x2x2, 2304 framework atoms) through
    rg_cbmc_external_energies, to 1e-6 K."""
    ff, cell, fw, atoms = static_co2_mfi_system()
    sysg = native.System(ctx, ff, cell, fw)
    sysg.set_molecules(atoms)
    trials = sysg.external_energies(atoms, 1)
    got = np.array([sum(t.framework_vdw for t in trials), sum(t.framework_charge for t in trials),
                    sum(t.molecule_vdw for t in trials[:3]), sum(t.molecule_charge for t in trials[:3])])
    np.testing.assert_allclose(got * ENERGY_TO_KELVIN, STATIC_CO2_MFI, rtol=0, atol=1e-6)
    sysg.close()


@pytest.fixture(scope="module")
def charged_box(ctx):
    """The charged synthetic framework in a 2x2x3 simulation box, FP64 grids on a 0.5 A mesh, 30 CO2."""
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


def test_first_bead_trials_grid_branch(charged_box, oracle):
    c = charged_box
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


def test_orientation_trials_with_skip(charged_box, oracle):
    """Chain-growth trial sets (three CO2 atoms around a fixed first bead, first bead skipped)."""
    c = charged_box
    ff = c["ff"]
    rng = np.random.default_rng(5)
    center = rng.random(3) @ c["scell"]
    sets = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, center, random_rotation(rng), 30) for _ in range(10)]
    trials = np.concatenate(sets)
    got = c["sys"].external_energies(trials, 3, skip=1)
    for t in range(10):
        ok, ref = oracle_trial(oracle, c, sets[t], skip=1)
        check(got[t], ok, ref)


def test_pair_loop_branch_fractional_and_groups(charged_box, oracle):
    """A fractional CFCMC molecule (no grid branch): framework pair loop over 3456 atoms, lambda 0.6, group 1."""
    c = charged_box
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


def test_skip_background_molecule(charged_box, oracle):
    c = charged_box
    ff = c["ff"]
    old = c["ads"][6:9]  # molecule 2, retraced: its own interactions are skipped by moleculeId
    trial = old.copy()
    got = c["sys"].external_energies(trial, 3, skip_background=2)
    ok, ref = oracle_trial(oracle, c, trial, skip_background=2)
    check(got[0], ok, ref)


def test_fp32c_trial_energies(charged_box, oracle):
    """RG_PRECISION_FP32C: Lennard-Jones pair terms in FP32 from the FP64 minimum-image displacement with
    TwoSum-compensated FP32 sums; the real-space Coulomb pairs and the grid branch in FP64. Bound: the trial's energy
    within 1e-6 of itself, and each part within 1e-6 of itself (both with a floor of 1 K where a sum crosses zero)."""
    c = charged_box
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
            kelvin = 1.0 / ENERGY_TO_KELVIN
            total = sum(getattr(g, k) for k in FIELDS)
            ref_total = sum(ref[k] for k in FIELDS)
            assert abs(total - ref_total) <= 1e-6 * max(kelvin, abs(ref_total)), (total, ref_total)
            for k in FIELDS:
                assert abs(getattr(g, k) - ref[k]) <= 1e-6 * max(kelvin, abs(ref[k])), (k, getattr(g, k), ref[k])
    assert n_ok >= 10


# ---- the energy differences of translation / rotation / CFCMC moves (B6) ----

DIFF_FIELDS = {"framework_vdw": "framework_molecule_vdw", "framework_charge": "framework_molecule_charge",
               "molecule_vdw": "molecule_molecule_vdw", "molecule_charge": "molecule_molecule_charge"}


def check_difference(gpu, ok, ref, fields, scale_extra=1.0):
    assert bool(gpu.overlap) == (not ok)
    if not ok:
        return
    for k in fields:
        r = ref[DIFF_FIELDS[k]]
        assert abs(getattr(gpu, k) - r) <= 1e-9 * max(scale_extra, abs(r)), (k, getattr(gpu, k), r)
    for g in range(4):
        for gk, rk in (("dudlambda_vdw", "dudlambda_vdw"), ("dudlambda_charge", "dudlambda_charge")):
            assert abs(getattr(gpu, gk)[g] - ref[rk][g]) <= 1e-9 * max(1.0, abs(ref[rk][g])), (gk, g)


def moved_molecules(c, seed, n=8, lam=1.0, fractional=False, step=0.8):
    """(new, old) atom sets: stored molecules translated and rotated about their centre."""
    rng = np.random.default_rng(seed)
    out = []
    for m in rng.choice(len(c["ads"]) // 3, size=n, replace=False):
        old = c["ads"][3 * m:3 * m + 3].copy()
        xyz = np.stack([old["x"], old["y"], old["z"]], 1)
        centre = xyz[1]
        new_xyz = (xyz - centre) @ random_rotation(rng).T + centre + rng.normal(size=3) * step
        new = old.copy()
        new["x"], new["y"], new["z"] = new_xyz[:, 0], new_xyz[:, 1], new_xyz[:, 2]
        if lam != 1.0 or fractional:
            from raspa3_b200.forcefield import lambda_scaling

            svdw, scoul = lambda_scaling(lam)
            new["scaling_vdw"], new["scaling_coulomb"] = svdw, scoul
            new["group_fractional"] = 1 | ((1 if fractional else 0) << 4)
        out.append((new, old))
    return out


def test_framework_energy_difference_translation_rotation(charged_box, oracle):
    """rg_framework_molecule_energy_difference against the oracle's restatement of
    Interactions::computeFrameworkMoleculeEnergyDifference: grid branch (Ewald charge method, integer molecules)."""
    c = charged_box
    c["sys"].set_precision(native.PRECISION_FP64)
    n_ok = n_overlap = 0
    # every stored molecule, moved by a small step: most random placements in this dense framework overlap, and both
    # outcomes are compared
    for new, old in moved_molecules(c, 41, n=len(c["ads"]) // 3, step=0.3):
        got = c["sys"].framework_energy_difference(new, old)
        ok, ref = oracle.framework_molecule_energy_difference(c["ff"], c["scell"], c["sfw"], new, old,
                                                              grids=c["grids"], grid_dims=c["dims"],
                                                              grid_cell=c["ucell"])
        check_difference(got, ok, ref, ("framework_vdw", "framework_charge"))
        n_ok += ok
        n_overlap += not ok
    assert n_ok >= 3 and n_overlap >= 1, (n_ok, n_overlap)


def test_framework_energy_difference_cfcmc_and_charge_method(charged_box, oracle):
    """A fractional molecule (CFCMC lambda move) takes the framework pair loop with dU/dlambda groups; a charge method
    other than Ewald turns the grid branch off (framework_molecule.cpp:145-146) and, with charges on, is unsupported."""
    c = charged_box
    ff = c["ff"]
    for new, old in moved_molecules(c, 42, n=4, lam=0.55, fractional=True):
        got = c["sys"].framework_energy_difference(new, old)
        ok, ref = oracle.framework_molecule_energy_difference(ff, c["scell"], c["sfw"], new, old, grids=c["grids"],
                                                              grid_dims=c["dims"], grid_cell=c["ucell"])
        check_difference(got, ok, ref, ("framework_vdw", "framework_charge"))
    with pytest.raises(native.RaspaGpuError):
        c["sys"].framework_energy_difference(c["ads"][:3], c["ads"][:3], charge_method=native.CHARGE_METHOD_COULOMB)
    # no charges: the Coulomb charge method is accepted and every atom takes the pair loop
    import copy

    ffq = copy.deepcopy(ff)
    ffq.use_charge = False
    sys2 = native.System(c["sys"].ctx, ffq, c["scell"], c["sfw"])
    try:
        for idx, g in enumerate(c["grids"]):
            if g is not None:
                sys2.set_grid(idx, c["ucell"], c["dims"], g)
        for new, old in moved_molecules(c, 43, n=3):
            got = sys2.framework_energy_difference(new, old, charge_method=native.CHARGE_METHOD_COULOMB)
            ok, ref = oracle.framework_molecule_energy_difference(ffq, c["scell"], c["sfw"], new, old,
                                                                  grids=c["grids"], grid_dims=c["dims"],
                                                                  grid_cell=c["ucell"], charge_method_ewald=False)
            check_difference(got, ok, ref, ("framework_vdw", "framework_charge"))
            pair_loop = oracle.framework_molecule_energy_difference(ffq, c["scell"], c["sfw"], new, old)[1]
            assert abs(ref["framework_molecule_vdw"] - pair_loop["framework_molecule_vdw"]) < 1e-12 * max(
                1.0, abs(pair_loop["framework_molecule_vdw"]))
    finally:
        sys2.close()


def test_framework_energy_difference_overlap_only_for_new_atoms(charged_box, oracle):
    c = charged_box
    ff = c["ff"]
    fw_atom = c["sfw"][c["sfw"]["type"] == ff.index("O")][0]
    # a stored molecule that does not overlap the framework where it stands
    empty = c["ads"][:0]
    m = next(m for m in range(len(c["ads"]) // 3) if oracle.framework_molecule_energy_difference(
        ff, c["scell"], c["sfw"], c["ads"][3 * m:3 * m + 3], empty, grids=c["grids"], grid_dims=c["dims"],
        grid_cell=c["ucell"])[0])
    old = c["ads"][3 * m:3 * m + 3].copy()
    new = old.copy()
    for k in "xyz":
        new[k] += fw_atom[k] - new[k][0] + np.array([0.0, 0.0, 0.0])
    got = c["sys"].framework_energy_difference(new, old)
    assert got.overlap == 1
    got = c["sys"].framework_energy_difference(old, new)  # the overlapping set as the old one is not tested
    assert got.overlap == 0


def test_intermolecular_energy_difference_and_update(charged_box, oracle):
    """rg_intermolecular_energy_difference against Interactions::computeInterMolecularEnergyDifference, then an
    accepted move written back with rg_system_update_molecules is seen by the next difference."""
    c = charged_box
    ff = c["ff"]
    moves = moved_molecules(c, 44)
    for new, old in moves:
        got = c["sys"].intermolecular_energy_difference(new, old)
        ok, ref = oracle.intermolecular_energy_difference(ff, c["scell"], c["ads"], new, old)
        check_difference(got, ok, ref, ("molecule_vdw", "molecule_charge"))
    new, old = next((n, o) for n, o in moves if oracle.intermolecular_energy_difference(ff, c["scell"], c["ads"], n,
                                                                                       o)[0])
    m = int(old["molecule_id"][0])
    updated = c["ads"].copy()
    updated[3 * m:3 * m + 3] = new
    c["sys"].update_molecules(3 * m, new)
    try:
        for new2, old2 in moved_molecules(c, 45, n=4):
            if int(old2["molecule_id"][0]) == m:
                continue
            old2 = updated[3 * int(old2["molecule_id"][0]):3 * int(old2["molecule_id"][0]) + 3]
            got = c["sys"].intermolecular_energy_difference(new2, old2)
            ok, ref = oracle.intermolecular_energy_difference(ff, c["scell"], updated, new2, old2)
            check_difference(got, ok, ref, ("molecule_vdw", "molecule_charge"))
    finally:
        c["sys"].update_molecules(3 * m, old)


# ---- blocked pockets, the external field and the dual-cutoff correction (B1) ----

def test_blocked_pockets(charged_box, oracle):
    """CBMC::insideBlockedPockets: pocket centres in unit-cell fractions, minimum image in the unit cell, radius scaled
    by the atom's VDW scaling; the trial is flagged 2 (dropped)."""
    c = charged_box
    ff = c["ff"]
    pockets = np.array([[0.5, 0.5, 0.5, 4.0], [0.1, 0.9, 0.2, 3.0]])
    rng = np.random.default_rng(51)
    first = make_atoms(rng.random((64, 3)) @ c["scell"], ff.index("C_co2"), 0.70, molecule_ids=np.full(64, 30))
    c["sys"].set_blocked_pockets(c["ucell"], pockets)
    try:
        got = c["sys"].external_energies(first, 1)
        n_blocked = 0
        for t in range(64):
            blocked = oracle.inside_blocked_pockets(c["ucell"], pockets, first[t:t + 1])
            n_blocked += blocked
            if blocked:
                assert got[t].overlap == 2
            else:
                ok, ref = oracle_trial(oracle, c, first[t:t + 1])
                check(got[t], ok, ref)
        assert 0 < n_blocked < 64
    finally:
        c["sys"].set_blocked_pockets(c["ucell"], np.zeros((0, 4)))
    assert all(g.overlap != 2 for g in c["sys"].external_energies(first, 1))


@pytest.mark.parametrize("surface,geometry", [(native.SURFACE_MULLER_BROWN, (5.0, 5.0, 0.0, 0.0)),
                                              (native.SURFACE_THIRD_ORDER_POLYNOMIAL, (5.0, 5.0, 0.0, 0.0)),
                                              (native.SURFACE_CYLINDER_Z, (9.0, 0.0, 0.0, 0.0)),
                                              (native.SURFACE_RECTANGLE_X, (8.0, 12.0, 0.0, 0.0)),
                                              (native.SURFACE_RECTANGLE_Z, (8.0, 12.0, 0.0, 0.0))])
def test_external_field_analytic(charged_box, oracle, surface, geometry):
    """CBMC::computeExternalFieldEnergy without a grid: the energy of each trial atom and the confinements that drop
    trials outside them."""
    c = charged_box
    ff = c["ff"]
    rng = np.random.default_rng(52)
    if surface == native.SURFACE_MULLER_BROWN:
        # the surface's own region (beyond it the exponentials overflow in both implementations)
        xyz = np.column_stack([rng.uniform(-1.5, 1.2, 48), rng.uniform(-0.5, 2.0, 48), rng.uniform(0, 10, 48)])
    else:
        xyz = rng.random((48, 3)) @ c["scell"]
    first = make_atoms(xyz, ff.index("C_co2"), 0.70, molecule_ids=np.full(48, 30))
    c["sys"].set_external_field(surface, geometry)
    try:
        got = c["sys"].external_energies(first, 1)
    finally:
        c["sys"].set_external_field(native.SURFACE_OFF)
    n_out = 0
    for t in range(48):
        ok_f, ef = oracle.external_field_energy(surface, geometry, c["scell"], first[t:t + 1])
        if not ok_f:
            n_out += 1
            assert got[t].overlap == 1
            continue
        ok, ref = oracle_trial(oracle, c, first[t:t + 1])
        check(got[t], ok, ref)
        assert abs(got[t].external_field_vdw - ef) <= 1e-12 * max(1.0, abs(ef)), (got[t].external_field_vdw, ef)
    if surface >= native.SURFACE_CYLINDER_X:
        assert 0 < n_out < 48


def test_external_field_grid(charged_box, oracle):
    """The external field from a tricubic grid over the simulation box, scaled by each atom's VDW scaling."""
    c = charged_box
    ff = c["ff"]
    dims = (17, 17, 18)
    grid, _ = c["sys"].ctx.grid_build(0, ff, c["scell"], c["sfw"], ff.index("C_co2"), 12.0, dims,
                                      native.PRECISION_FP64)
    rng = np.random.default_rng(53)
    sets = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 31, lam=0.7,
                           group=1, fractional=True) for _ in range(8)]
    c["sys"].set_external_field(native.SURFACE_GRID_FILE, grid=grid, grid_cell=c["scell"], grid_dims=dims)
    try:
        got = c["sys"].external_energies(np.concatenate(sets), 3, skip=2)
    finally:
        c["sys"].set_external_field(native.SURFACE_OFF)
    for t in range(8):
        ok_f, ef = oracle.external_field_energy(native.SURFACE_GRID_FILE, (0, 0, 0, 0), c["scell"], sets[t],
                                                grid=grid, grid_dims=dims, grid_cell=c["scell"], skip=2)
        assert ok_f
        assert abs(got[t].external_field_vdw - ef) <= 1e-9 * max(1.0, abs(ef)), (got[t].external_field_vdw, ef)


def test_dual_cutoff_correction(charged_box, oracle):
    """CBMC::computeDualCutOffCorrection: the set's energy with the force field's cutoffs minus with the dual cutoff,
    pair-loop (fractional) and grid-branch sets alike."""
    c = charged_box
    ff = c["ff"]
    rng = np.random.default_rng(54)
    sets = [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 31, lam=0.8,
                           group=1, fractional=True) for _ in range(3)]
    sets += [rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ c["scell"], random_rotation(rng), 31)
             for _ in range(3)]
    dual = 7.5
    for s in sets:
        got = c["sys"].dual_cutoff_correction(s, dual)
        okf, ef = oracle.cbmc_framework_molecule(ff, c["scell"], c["sfw"], s, ff.cutoff_framework_vdw,
                                                 ff.cutoff_coulomb, grids=c["grids"], grid_dims=c["dims"],
                                                 grid_cell=c["ucell"])
        oki, ei = oracle.cbmc_framework_molecule(ff, c["scell"], c["sfw"], s, dual, dual, grids=c["grids"],
                                                 grid_dims=c["dims"], grid_cell=c["ucell"])
        okm, em = oracle.cbmc_intermolecular(ff, c["scell"], c["ads"], s, ff.cutoff_molecule_vdw, ff.cutoff_coulomb)
        okn, en = oracle.cbmc_intermolecular(ff, c["scell"], c["ads"], s, dual, dual)
        ok = okf and oki and okm and okn
        assert bool(got.overlap) == (not ok)
        if not ok:
            continue
        for k in FIELDS:
            ref = (ef[ORACLE[k]] + em[ORACLE[k]]) - (ei[ORACLE[k]] + en[ORACLE[k]])
            assert abs(getattr(got, k) - ref) <= 1e-9 * max(1.0, abs(ef[ORACLE[k]]) + abs(em[ORACLE[k]])), (k,)

"""(c) Ewald Fourier path on the GPU through the C-ABI vs the FP64 oracle and the reference goldens."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ENERGY_TO_KELVIN
from raspa3_b200.synthetic import (CO2_NAMES, CO2_OFFSETS, random_molecules, random_rotation, rigid_molecule,
                                   synthetic_forcefield, synthetic_framework)
from reference_systems import co2_atoms, itq29, mfi, zeolite_forcefield

pytestmark = pytest.mark.gpu

TERMS = ("ewald_fourier", "ewald_self", "ewald_exclusion")


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def total(e):
    return sum(e[k] for k in TERMS)


def test_golden_two_co2_in_10A_box(ctx):
    """tests/raspakit-tests/ewald.cpp:25-54 -> 90.54613836 K (full half-box k-set, alpha 0.25, kmax 8)."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    cell = np.diag([10.0, 10.0, 10.0])
    ew = native.Ewald(ctx, ff, cell)
    assert ew.n_kvectors == 2600
    atoms = co2_atoms(ff, [(-1.0, 0.0, 0.0), (1.0, 0.0, 0.0)], [0, 1])
    e = ew.full(atoms, [3, 3])
    assert abs(total(e) * ENERGY_TO_KELVIN - 90.54613836) < 1e-6


@pytest.mark.parametrize("rep,single_ion,fourier", [((1, 1, 1), 17464.2371790130, -702.65863478),
                                                    ((2, 2, 2), 9673.9032373025, -721.64644486)])
def test_golden_itq29_with_framework(ctx, rep, single_ion, fourier):
    """tests/raspakit-tests/ewald.cpp:146-210."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    cell, fw = itq29(ff, rep)
    ew = native.Ewald(ctx, ff, cell)
    ew.set_framework(fw)
    c = 5.93355
    atoms = co2_atoms(ff, [(c, 7.93355, c), (c, 3.93355, c)], [0, 1])
    e = ew.full(atoms, [3, 3])
    assert abs(total(e) * ENERGY_TO_KELVIN - fourier) < 1e-6
    # the single-ion sum of the unit charge (ewald.cpp:210-274) from the k-table: -C(2pi/V sum' - alpha/sqrt(pi))
    import math
    from raspa3_b200.forcefield import COULOMBIC_CONVERSION_FACTOR as C
    u = -(ew.single_ion_sum - C * ff.ewald_alpha / math.sqrt(math.pi))
    assert abs(u * ENERGY_TO_KELVIN - single_ion) < 1e-6


@pytest.mark.parametrize("rep,single_ion,fourier", [((1, 1, 1), 12028.1731827280, -1191.77790165),
                                                    ((2, 2, 2), 6309.7866899037, -1197.23909965)])
def test_golden_mfi_with_framework(ctx, rep, single_ion, fourier):
    """tests/raspakit-tests/ewald.cpp:212-278: 2 CO2 in MFI (Framework::makeMFI, P n m a) 1x1x1 and 2x2x2."""
    import math
    from raspa3_b200.forcefield import COULOMBIC_CONVERSION_FACTOR as C

    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    cell, fw = mfi(ff, rep)
    ew = native.Ewald(ctx, ff, cell)
    ew.set_framework(fw)
    atoms = co2_atoms(ff, [(10.011, 4.97475 + 2.0, 0.0), (10.011, 4.97475 - 2.0, 0.0)], [0, 1])
    e = ew.full(atoms, [3, 3])
    assert abs(total(e) * ENERGY_TO_KELVIN - fourier) < 1e-6
    u = -(ew.single_ion_sum - C * ff.ewald_alpha / math.sqrt(math.pi))
    assert abs(u * ENERGY_TO_KELVIN - single_ion) < 1e-6
    ew.close()


def charged_co2_box(n_mol=24, seed=3, sphere=True):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8, sphere=sphere)
    cell, fw = synthetic_framework(ff, seed=42)
    ads = random_molecules(ff, cell, n_mol, seed=seed)
    return ff, cell, fw, ads


@pytest.mark.parametrize("sphere,nk", [(True, 1152), (False, 2600)])
def test_kvector_counts_charged_co2_box(ctx, oracle, sphere, nk):
    ff, cell, fw, ads = charged_co2_box(sphere=sphere)
    ew = native.Ewald(ctx, ff, cell)
    kv, temp, s = oracle.ewald_kvectors(ff, cell)
    assert ew.n_kvectors == nk == len(kv)
    assert abs(ew.single_ion_sum - s) <= 1e-12 * abs(s)


def test_full_and_delta_match_oracle(ctx, oracle):
    ff, cell, fw, ads = charged_co2_box()
    ew = native.Ewald(ctx, ff, cell, n_groups=0)
    ew.set_framework(fw)
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    np.testing.assert_allclose(ew.structure_factors(2), s_rigid, rtol=0, atol=1e-9 * np.max(np.abs(s_rigid)))
    sizes = [3] * (len(ads) // 3)
    e_gpu = ew.full(ads, sizes)
    e_ref, stored = oracle.ewald_fourier_energy(ff, cell, ads, sizes, s_rigid=s_rigid)
    for k in TERMS:
        assert abs(e_gpu[k] - e_ref[k]) <= 1e-9 * max(1.0, abs(e_ref[k])), k
    rng = np.random.default_rng(5)
    for trial in range(20):
        m = int(rng.integers(len(sizes)))
        old = ads[3 * m: 3 * m + 3]
        new = old.copy()
        shift = rng.normal(size=3)
        for i, k in enumerate("xyz"):
            new[k] += shift[i]
        d_gpu = ew.delta(new, old)
        d_ref, trial_ref = oracle.ewald_delta(ff, cell, stored, new, old)
        scale = max(1.0, abs(d_ref["ewald_fourier"]))
        for k in TERMS:
            assert abs(d_gpu[k] - d_ref[k]) <= 1e-6 * scale, (k, d_gpu[k], d_ref[k])
        t_gpu = ew.structure_factors(1)
        np.testing.assert_allclose(t_gpu[0::2], trial_ref[0::10], rtol=0, atol=1e-9)
        np.testing.assert_allclose(t_gpu[1::2], trial_ref[1::10], rtol=0, atol=1e-9)


def test_insertion_and_deletion_deltas(ctx, oracle):
    ff, cell, fw, ads = charged_co2_box()
    ew = native.Ewald(ctx, ff, cell)
    ew.set_framework(fw)
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    sizes = [3] * (len(ads) // 3)
    ew.full(ads, sizes)
    _, stored = oracle.ewald_fourier_energy(ff, cell, ads, sizes, s_rigid=s_rigid)
    rng = np.random.default_rng(9)
    ins = rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ cell, random_rotation(rng), 999)
    empty = ins[:0]
    for new, old in ((ins, empty), (empty, ads[:3])):
        d_gpu = ew.delta(new, old)
        d_ref, _ = oracle.ewald_delta(ff, cell, stored, new, old)
        for k in TERMS:
            assert abs(d_gpu[k] - d_ref[k]) <= 1e-6 * max(1.0, abs(d_ref[k])), k


def test_fractional_molecule_dudlambda_groups(ctx, oracle):
    """A CFCMC fractional molecule (lambda = 0.7, group 1): dU/dlambda group sums (ewald.cpp:166-173, 1221-1238)."""
    ff, cell, fw, ads = charged_co2_box(n_mol=10)
    rng = np.random.default_rng(2)
    frac = rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ cell, random_rotation(rng), 500, lam=0.7,
                          group=1, fractional=True)
    allatoms = np.concatenate([ads, frac])
    sizes = [3] * (len(allatoms) // 3)
    ew = native.Ewald(ctx, ff, cell, n_groups=4)
    ew.set_framework(fw)
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    e_gpu = ew.full(allatoms, sizes)
    e_ref, stored = oracle.ewald_fourier_energy(ff, cell, allatoms, sizes, s_rigid=s_rigid)
    np.testing.assert_allclose(e_gpu["dudlambda_ewald"], e_ref["dudlambda_ewald"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(ew.structure_factors(0), stored, rtol=0, atol=1e-9)
    new = frac.copy()
    for k in "xyz":
        new[k] += 0.4
    d_gpu = ew.delta(new, frac)
    d_ref, _ = oracle.ewald_delta(ff, cell, stored, new, frac)
    np.testing.assert_allclose(d_gpu["dudlambda_ewald"], d_ref["dudlambda_ewald"], rtol=1e-7, atol=1e-7)
    for k in TERMS:
        assert abs(d_gpu[k] - d_ref[k]) <= 1e-6 * max(1.0, abs(d_ref[k])), k


def test_running_energy_drift_over_many_moves(ctx, oracle):
    """Running sum of accepted deltas vs a full recompute after 300 moves (the reference drift tests,
    tests/raspa3-tests/mc_*_drift.cpp, require < 1e-6 per term)."""
    ff, cell, fw, ads = charged_co2_box(n_mol=30, seed=4)
    ew = native.Ewald(ctx, ff, cell)
    ew.set_framework(fw)
    sizes = [3] * (len(ads) // 3)
    running = total(ew.full(ads, sizes))
    rng = np.random.default_rng(11)
    ads = ads.copy()
    for step in range(300):
        m = int(rng.integers(len(sizes)))
        old = ads[3 * m: 3 * m + 3].copy()
        new = rigid_molecule(ff, CO2_NAMES, CO2_OFFSETS, rng.random(3) @ cell, random_rotation(rng), m)
        d = ew.delta(new, old)
        if rng.random() < 0.5:
            ew.accept()
            running += total(d)
            ads[3 * m: 3 * m + 3] = new
    s_gpu = ew.structure_factors(0)
    recomputed = total(ew.full(ads, sizes))
    assert abs(running - recomputed) < 1e-6 * max(1.0, abs(recomputed))
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    e_ref, stored = oracle.ewald_fourier_energy(ff, cell, ads, sizes, s_rigid=s_rigid)
    assert abs(recomputed - total(e_ref)) < 1e-8 * max(1.0, abs(total(e_ref)))
    np.testing.assert_allclose(s_gpu[0::2], stored[0::10], rtol=0, atol=1e-8)


@pytest.mark.parametrize("kmax,sphere", [(12, False), (9, True)])
def test_batched_structure_factor_update(ctx, oracle, kmax, sphere):
    """rg_ewald_batch: one CO2 move in each of 40 systems that share one set of k-vectors, in one launch: the
    large-mixture set (kmax 12, the full half-box, 8,124 k-vectors) with translations, and a spherical set (kmax 9, runs of kz of
    every length) with insertions, deletions and translations. Each system's Fourier energy change and trial S(k)
    equal the oracle's energyDifferenceEwaldFourier on that system's own S(k) (1e-9), and accepting flips only the
    accepted systems."""
    from raspa3_b200.synthetic import random_molecules

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=kmax, sphere=sphere)
    cell = np.diag([40.0, 39.8, 40.2])
    ew = native.Ewald(ctx, ff, cell)
    nk = ew.n_kvectors
    n_sys = 40
    batch = native.EwaldBatch(ew, n_sys)
    rng = np.random.default_rng(12)
    oracle_stored, moves = [], []
    for s in range(n_sys):
        mols = random_molecules(ff, cell, 20, seed=100 + s)
        ew.full(mols, [3] * 20)  # this system's structure factor into the Ewald state, then into the batch
        batch.set(s)
        _, so = oracle.ewald_fourier_energy(ff, cell, mols, [3] * 20)
        oracle_stored.append(so)
        np.testing.assert_allclose(batch.get(s, 0)[0::2], so[0::10][:nk], rtol=0, atol=1e-9)
        old = mols[3 * (s % 20):3 * (s % 20) + 3]
        new = old.copy()
        for k in "xyz":
            new[k] += rng.normal() * 0.6
        kind = s % 3 if sphere else 2
        moves.append((new if kind != 1 else new[:0], old if kind != 0 else old[:0]))
    packed = np.zeros(6 * n_sys, dtype=moves[0][1].dtype if len(moves[0][1]) else moves[0][0].dtype)
    for s, (new, old) in enumerate(moves):
        packed[6 * s:6 * s + len(new)] = new
        packed[6 * s + len(new):6 * s + len(new) + len(old)] = old
    d = batch.delta(packed, 6, [len(m[0]) for m in moves], [len(m[1]) for m in moves])
    upload_ms, kernel_ms = batch.timing()
    assert upload_ms >= 0.0 and kernel_ms > 0.0, (upload_ms, kernel_ms)
    trials = []
    for s in range(n_sys):
        new, old = moves[s]
        ref, trial = oracle.ewald_delta(ff, cell, oracle_stored[s], new, old)
        trials.append(trial)
        assert abs(d[s] - ref["ewald_fourier"]) <= 1e-9 * max(1.0, abs(ref["ewald_fourier"])), (s, d[s], ref)
        got_trial = batch.get(s, 1)
        np.testing.assert_allclose(got_trial[0::2], trial[0::10][:nk], rtol=0, atol=1e-9)
        np.testing.assert_allclose(got_trial[1::2], trial[1::10][:nk], rtol=0, atol=1e-9)
    mask = np.arange(n_sys) % 3 == 0
    batch.accept(mask)
    for s in range(6):
        now = batch.get(s, 0)
        ref = trials[s] if mask[s] else oracle_stored[s]
        np.testing.assert_allclose(now[0::2], ref[0::10][:nk], rtol=0, atol=1e-9)
        np.testing.assert_allclose(now[1::2], ref[1::10][:nk], rtol=0, atol=1e-9)
    batch.close()
    ew.close()

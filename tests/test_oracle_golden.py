"""The FP64 oracle against RASPA3's own known-answer tests (the pins of every parity claim)."""

import numpy as np
import pytest

from raspa3_b200.forcefield import ENERGY_TO_KELVIN, COULOMBIC_CONVERSION_FACTOR, make_atoms
from reference_systems import ITQ29_A, auto_ewald_alpha, co2_atoms, itq29, methane_atoms, mfi, zeolite_forcefield


def test_units_match_reference_constants(oracle):
    assert oracle.energy_to_kelvin() == ENERGY_TO_KELVIN
    assert oracle.lib().oracle_coulomb_factor() == COULOMBIC_CONVERSION_FACTOR
    # units.cpp documents EnergyToKelvin ~ 1.2027242847 and the Coulomb constant 138935.4835 (internal units)
    assert abs(ENERGY_TO_KELVIN - 1.2027242847) < 1e-9
    assert abs(COULOMBIC_CONVERSION_FACTOR - 138935.4835) < 1e-3


def test_ewald_two_co2_in_10A_box(oracle):
    """tests/raspakit-tests/ewald.cpp:25-54: Fourier + self + exclusion = 90.54613836 K."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    ff.kmax = (8, 8, 8)
    cell = np.diag([10.0, 10.0, 10.0])
    atoms = co2_atoms(ff, [(-1.0, 0.0, 0.0), (1.0, 0.0, 0.0)], [0, 1])
    e, stored = oracle.ewald_fourier_energy(ff, cell, atoms, [3, 3])
    total = (e["ewald_fourier"] + e["ewald_self"] + e["ewald_exclusion"]) * ENERGY_TO_KELVIN
    assert abs(total - 90.54613836) < 1e-6


def test_itq29_expansion_counts():
    ff = zeolite_forcefield()
    cell, atoms = itq29(ff)
    assert len(atoms) == 72
    assert int(np.sum(atoms["type"] == ff.index("Si"))) == 24
    assert abs(float(np.sum(atoms["charge"]))) < 1e-12


def test_framework_molecule_methane_itq29(oracle):
    """tests/raspakit-tests/cbmc_interactions.cpp:27-51: -337.77056357 K."""
    ff = zeolite_forcefield(12.0, True, use_charge=False)
    cell, fw = itq29(ff)
    m = methane_atoms(ff, [(0.5 * ITQ29_A, 0.5 * ITQ29_A, 0.5 * ITQ29_A)], [0])
    ok, e = oracle.cbmc_framework_molecule(ff, cell, fw, m, 12.0, 12.0)
    assert ok
    assert abs(e["framework_molecule_vdw"] * ENERGY_TO_KELVIN - (-337.77056357)) < 1e-6


def test_framework_and_intermolecular_two_methanes_itq29(oracle):
    """tests/raspakit-tests/cbmc_interactions.cpp:53-90: -1599.10322574 K and 2352.42793591 K."""
    ff = zeolite_forcefield(12.0, True, use_charge=False)
    cell, fw = itq29(ff)
    a = ITQ29_A
    m = methane_atoms(ff, [(0.5 * a, 0.5 * a, 0.5 * a), (0.6 * a, 0.7 * a, 0.65 * a)], [0, 1])
    ok, e = oracle.cbmc_framework_molecule(ff, cell, fw, m, 12.0, 12.0)
    assert ok
    assert abs(e["framework_molecule_vdw"] * ENERGY_TO_KELVIN - (-1599.10322574)) < 1e-6
    ok1, e1 = oracle.cbmc_intermolecular(ff, cell, m, m[:1], 12.0, 12.0)
    ok2, e2 = oracle.cbmc_intermolecular(ff, cell, m, m[1:], 12.0, 12.0)
    ok3, e3 = oracle.cbmc_intermolecular(ff, cell, m, m, 12.0, 12.0)
    assert ok1 and ok2 and ok3
    assert abs(e1["molecule_molecule_vdw"] * ENERGY_TO_KELVIN - 2352.42793591) < 1e-6
    assert abs(e2["molecule_molecule_vdw"] * ENERGY_TO_KELVIN - 2352.42793591) < 1e-6
    assert abs(e3["molecule_molecule_vdw"] * ENERGY_TO_KELVIN / 2.0 - 2352.42793591) < 1e-6


# tests/raspakit-tests/static_energy.cpp:21-46: framework VDW, framework charge, molecule VDW, molecule charge (K)
STATIC_CO2_ITQ29 = (-1545.62921755, -592.13188606, -242.42459776, 154.11883595)


def static_co2_itq29_system():
    """2 CO2 in ITQ-29 1x1x1 with the zeolite force field, charges on and the automatic Ewald alpha that the reference's
    System sets (static_energy.cpp:21-46)."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = auto_ewald_alpha(12.0)
    cell, fw = itq29(ff)
    c = 5.93355
    atoms = co2_atoms(ff, [(c, 7.93355, c), (c, 3.93355, c)], [0, 1])
    return ff, cell, fw, atoms


def test_static_energy_two_co2_in_itq29(oracle):
    """The real-space Coulomb pair (potentialCoulomb<0>, Ewald) against the framework and between molecules, pinned
    to the reference's charged golden: all four energy terms to 1e-6 K."""
    ff, cell, fw, atoms = static_co2_itq29_system()
    assert abs(ff.ewald_alpha - 0.26505830360350674) < 1e-15
    ok, e = oracle.cbmc_framework_molecule(ff, cell, fw, atoms, 12.0, 12.0)
    ok2, e2 = oracle.cbmc_intermolecular(ff, cell, atoms, atoms[:3], 12.0, 12.0)
    assert ok and ok2
    got = (e["framework_molecule_vdw"], e["framework_molecule_charge"], e2["molecule_molecule_vdw"],
           e2["molecule_molecule_charge"])
    for g, ref in zip(got, STATIC_CO2_ITQ29):
        assert abs(g * ENERGY_TO_KELVIN - ref) < 1e-6, (g * ENERGY_TO_KELVIN, ref)


@pytest.mark.parametrize("rep,single_ion,fourier", [
    ((1, 1, 1), 17464.2371790130, -702.65863478),
    ((2, 2, 2), 9673.9032373025, -721.64644486),
])
def test_ewald_two_co2_in_itq29(oracle, rep, single_ion, fourier):
    """tests/raspakit-tests/ewald.cpp:146-210: single-ion Fourier sum and Fourier+self+exclusion with the rigid
    framework structure factor subtracted."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    ff.kmax = (8, 8, 8)
    cell, fw = itq29(ff, rep)
    c = 5.93355
    atoms = co2_atoms(ff, [(c, 7.93355, c), (c, 3.93355, c)], [0, 1])
    assert abs(oracle.ewald_single_ion(ff, cell, (0.0, 0.0, 0.0), 1.0) * ENERGY_TO_KELVIN - single_ion) < 1e-6
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    e, _ = oracle.ewald_fourier_energy(ff, cell, atoms, [3, 3], s_rigid=s_rigid)
    total = (e["ewald_fourier"] + e["ewald_self"] + e["ewald_exclusion"]) * ENERGY_TO_KELVIN
    assert abs(total - fourier) < 1e-6


def test_ewald_delta_equals_difference_of_full_sums(oracle):
    """energyDifferenceEwaldFourier (ewald.cpp:1043-1244) == E(new) - E(old) of computeEwaldFourierEnergy, the
    property behind the reference's drift tests (tests/raspa3-tests/mc_*_drift.cpp)."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    cell, fw = itq29(ff, (1, 1, 1))
    c = 5.93355
    old = co2_atoms(ff, [(c, 7.93355, c), (c, 3.93355, c)], [0, 1])
    new = old.copy()
    for k in "xyz":
        new[k][3:] += 0.37
    s_rigid = oracle.ewald_rigid(ff, cell, fw)
    e_old, stored = oracle.ewald_fourier_energy(ff, cell, old, [3, 3], s_rigid=s_rigid)
    e_new, stored_new = oracle.ewald_fourier_energy(ff, cell, new, [3, 3], s_rigid=s_rigid)
    d, trial = oracle.ewald_delta(ff, cell, stored, new[3:], old[3:])
    full = sum(e_new[k] - e_old[k] for k in ("ewald_fourier", "ewald_self", "ewald_exclusion"))
    delta = d["ewald_fourier"] + d["ewald_self"] + d["ewald_exclusion"]
    assert abs(full - delta) < 1e-8 * max(1.0, abs(full))
    np.testing.assert_allclose(trial[0::10], stored_new[0::10], rtol=0, atol=1e-10)


def test_energy_differences_are_differences_of_energies(oracle):
    """The oracle's restatements of computeFrameworkMoleculeEnergyDifference and computeInterMolecularEnergyDifference
    (pair-loop branch) equal E(new) - E(old) of the CBMC energies, for a charged framework and two CO2."""
    ff, cell, fw, atoms = static_co2_itq29_system()
    new = atoms[3:].copy()
    for k, d in zip("xyz", (0.31, -0.2, 0.44)):
        new[k] += d
    old = atoms[3:]
    ok, d = oracle.framework_molecule_energy_difference(ff, cell, fw, new, old)
    ok_n, e_n = oracle.cbmc_framework_molecule(ff, cell, fw, new, 12.0, 12.0)
    ok_o, e_o = oracle.cbmc_framework_molecule(ff, cell, fw, old, 12.0, 12.0)
    assert ok and ok_n and ok_o
    for k in ("framework_molecule_vdw", "framework_molecule_charge"):
        assert abs(d[k] - (e_n[k] - e_o[k])) < 1e-10 * max(1.0, abs(e_n[k]))
    ok, d = oracle.intermolecular_energy_difference(ff, cell, atoms, new, old)
    ok_n, e_n = oracle.cbmc_intermolecular(ff, cell, atoms, new, 12.0, 12.0)
    ok_o, e_o = oracle.cbmc_intermolecular(ff, cell, atoms, old, 12.0, 12.0)
    assert ok and ok_n and ok_o
    for k in ("molecule_molecule_vdw", "molecule_molecule_charge"):
        assert abs(d[k] - (e_n[k] - e_o[k])) < 1e-10 * max(1.0, abs(e_n[k]))
    # omitInterInteractions: no intermolecular difference at all (intermolecular.cpp:207)
    ff.omit_inter = True
    ok, d = oracle.intermolecular_energy_difference(ff, cell, atoms, new, old)
    assert ok and d["molecule_molecule_vdw"] == 0.0 and d["molecule_molecule_charge"] == 0.0


def test_blocked_pockets_and_external_field_oracle(oracle):
    """insideBlockedPockets: minimum image in the unit cell, radius scaled by sqrt(scalingVDW); external field: the
    reference's Muller-Brown parameter set (interactions_external_field.cpp:68-78, whose fourth amplitude is -15
    where the published surface has +15) evaluated independently here, and a confining cylinder."""
    cell = np.diag([10.0, 12.0, 14.0])
    a = make_atoms([(9.8, 0.1, 0.2)], 0, 0.0)
    assert oracle.inside_blocked_pockets(cell, [(0.0, 0.0, 0.0, 1.0)], a)  # across the periodic boundary
    assert not oracle.inside_blocked_pockets(cell, [(0.5, 0.5, 0.5, 1.0)], a)
    a["scaling_vdw"] = 0.01  # radius 0.1: the atom at 0.3 A is outside
    assert not oracle.inside_blocked_pockets(cell, [(0.0, 0.0, 0.0, 1.0)], a)
    import math

    amp, a_, x0, b_, y0, c_ = ((-200.0, -100.0, -170.0, -15.0), (-1.0, -1.0, -6.5, -0.7), (1.0, 0.0, -0.5, -1.0),
                               (0.0, 0.0, 11.0, 0.6), (0.0, 0.5, 1.5, 1.0), (-10.0, -10.0, -6.5, 0.7))
    x, y = -0.558, 1.442
    expect = sum(amp[i] * math.exp(a_[i] * (x - x0[i]) ** 2 + b_[i] * (x - x0[i]) * (y - y0[i]) +
                                   c_[i] * (y - y0[i]) ** 2) for i in range(4))
    ok, e = oracle.external_field_energy(8, (5, 5, 0, 0), cell, make_atoms([(x, y, 0.0)], 0, 0.0))
    assert ok and abs(e - expect) < 1e-12 * abs(expect)
    ok, e = oracle.external_field_energy(13, (2.0, 0, 0, 0), cell, make_atoms([(5.5, 6.5, 100.0)], 0, 0.0))
    assert ok and e == 0.0  # 0.71 A from the z axis through the box centre (the position is not wrapped)
    ok, _ = oracle.external_field_energy(13, (2.0, 0, 0, 0), cell, make_atoms([(5.0, 9.0, 1.0)], 0, 0.0))
    assert not ok


def test_mfi_expansion_counts():
    """Framework::makeMFI: 12 Si + 26 O in the asymmetric unit, P n m a -> 96 Si + 192 O, neutral."""
    ff = zeolite_forcefield()
    cell, atoms = mfi(ff)
    assert len(atoms) == 288 and int(np.sum(atoms["type"] == ff.index("Si"))) == 96
    assert abs(float(np.sum(atoms["charge"]))) < 1e-9
    np.testing.assert_allclose(np.diag(cell), (20.022, 19.899, 13.383))


@pytest.mark.parametrize("rep,single_ion,fourier", [
    ((1, 1, 1), 12028.1731827280, -1191.77790165),
    ((2, 2, 2), 6309.7866899037, -1197.23909965),
])
def test_ewald_two_co2_in_mfi(oracle, rep, single_ion, fourier):
    """tests/raspakit-tests/ewald.cpp:212-278."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = 0.25
    ff.kmax = (8, 8, 8)
    cell, fw = mfi(ff, rep)
    atoms = co2_atoms(ff, [(10.011, 4.97475 + 2.0, 0.0), (10.011, 4.97475 - 2.0, 0.0)], [0, 1])
    assert abs(oracle.ewald_single_ion(ff, cell, (0.0, 0.0, 0.0), 1.0) * ENERGY_TO_KELVIN - single_ion) < 1e-6
    e, _ = oracle.ewald_fourier_energy(ff, cell, atoms, [3, 3], s_rigid=oracle.ewald_rigid(ff, cell, fw))
    assert abs((e["ewald_fourier"] + e["ewald_self"] + e["ewald_exclusion"]) * ENERGY_TO_KELVIN - fourier) < 1e-6


# tests/raspakit-tests/static_energy.cpp:48-74: 2 CO2 in MFI 2x2x2, shifted
STATIC_CO2_MFI = (-2525.36580663, 2167.45591472, -242.42459776, 154.11883595)


def static_co2_mfi_system():
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    ff.ewald_alpha = auto_ewald_alpha(12.0)
    cell, fw = mfi(ff, (2, 2, 2))
    atoms = co2_atoms(ff, [(10.011, 4.97475 + 2.0, 0.0), (10.011, 4.97475 - 2.0, 0.0)], [0, 1])
    return ff, cell, fw, atoms


def test_static_energy_two_co2_in_mfi(oracle):
    ff, cell, fw, atoms = static_co2_mfi_system()
    ok, e = oracle.cbmc_framework_molecule(ff, cell, fw, atoms, 12.0, 12.0)
    ok2, e2 = oracle.cbmc_intermolecular(ff, cell, atoms, atoms[:3], 12.0, 12.0)
    assert ok and ok2
    got = (e["framework_molecule_vdw"], e["framework_molecule_charge"], e2["molecule_molecule_vdw"],
           e2["molecule_molecule_charge"])
    for g, ref in zip(got, STATIC_CO2_MFI):
        assert abs(g * ENERGY_TO_KELVIN - ref) < 1e-6, (g * ENERGY_TO_KELVIN, ref)

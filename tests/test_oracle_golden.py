"""The FP64 oracle against RASPA3's own known-answer tests (the pins of every parity claim)."""

import numpy as np
import pytest

from raspa3_b200.forcefield import ENERGY_TO_KELVIN, COULOMBIC_CONVERSION_FACTOR, make_atoms
from reference_systems import ITQ29_A, co2_atoms, itq29, methane_atoms, zeolite_forcefield


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

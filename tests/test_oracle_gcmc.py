"""The CPU GCMC oracle: acceptance rules checked against exact statistical mechanics."""

import numpy as np

from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, methane_component
from raspa3_b200.synthetic import synthetic_forcefield


def test_ideal_gas_loading_is_beta_f_v(oracle):
    """With every interaction switched off, CBMC swap moves must sample the Poisson distribution <N> = beta f V
    (the insertion / deletion Pacc of insertion_cbmc.cpp:158-168 and deletion_cbmc.cpp:157-161)."""
    ff = synthetic_forcefield(charges=False)
    for p in ff.pseudo_atoms:
        p.epsilon_k = 0.0
    ff.__post_init__()
    cell = np.diag([30.0, 30.0, 30.0])
    beta, f = beta_of(300.0), fugacity_of(2e5)
    expected = beta * f * 27000.0
    res, secs = oracle.gcmc_run(ff, cell, co2_component(), beta, f, n_chains=8, steps=20000, equilibration=2000,
                                use_ewald=False, threads=8)
    means = np.array([r["sum_n"] / r["samples"] for r in res])
    var = np.array([r["sum_n2"] / r["samples"] for r in res]) - means ** 2
    m, err = means.mean(), means.std(ddof=1) / np.sqrt(len(means))
    assert abs(m - expected) < 4 * err + 0.02 * expected, (m, err, expected)
    # Poisson: variance equals the mean
    assert abs(var.mean() - expected) < 0.15 * expected
    for r in res:
        assert abs(r["running_energy"] - r["recomputed_energy"]) < 1e-9


def test_drift_lj_fluid_in_box(oracle):
    """Methane fluid without framework at 300 K and 5 MPa: running vs recomputed energy (drift < 1e-6 relative)."""
    ff = synthetic_forcefield(charges=False)
    cell = np.diag([25.0, 25.0, 25.0])
    res, _ = oracle.gcmc_run(ff, cell, methane_component(), beta_of(300.0), fugacity_of(5e6), n_chains=2, steps=5000,
                             use_ewald=False, threads=2)
    for r in res:
        assert r["n_molecules"] > 5
        assert abs(r["running_energy"] - r["recomputed_energy"]) <= 1e-6 * max(1.0, abs(r["recomputed_energy"]))


def test_drift_co2_with_ewald_and_framework_grids(oracle):
    """CO2 in the charged synthetic framework (coarse FP64 grids from the oracle, framework S(k)) at 1 MPa:
    running vs recomputed energy after a few thousand moves, all move types accepted at least once."""
    from raspa3_b200.synthetic import replicate, synthetic_framework

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=6)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (21, 21, 15)
    grids = [None] * (ff.n_types + 1)
    for idx, gt in ((ff.index("C_co2"), 0), (ff.index("O_co2"), 0), (ff.n_types, 1)):
        grids[idx] = oracle.make_grid(gt, ff, ucell, ufw, idx if gt == 0 else 0, 12.0, dims, threads=8)
    s_fw = oracle.ewald_rigid(ff, scell, sfw)
    res, _ = oracle.gcmc_run(ff, scell, co2_component(), beta_of(300.0), fugacity_of(1e6), n_chains=2, steps=3000,
                             grids=grids, grid_dims=dims, grid_cell=ucell, s_framework=s_fw, threads=2, seed=3)
    for r in res:
        assert r["n_molecules"] >= 1
        assert min(r["accepted"]) >= 1, r["accepted"]
        assert abs(r["running_energy"] - r["recomputed_energy"]) <= 1e-6 * max(1.0, abs(r["recomputed_energy"]))

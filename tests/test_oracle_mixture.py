"""The CPU oracle of the mixture GCMC with identity change (oracle/mixture.cpp).

* Ideal-gas mixture (no framework, no intermolecular pairs, no Ewald): with translation, rotation, CBMC swap and
  identity change, <N_c> = beta f_c V for every component (the identity-change acceptance rule of
  mc_moves/component/identity_change.cpp:229-240 conserves the grand-canonical distribution).
* A small mixture in the synthetic framework (framework charges off, CO2 / N2 charged, Ewald on): the running energy
  equals the energy recomputed from scratch.
"""

import math

import numpy as np

from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, n2_component
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

BETA = beta_of(300.0)


def test_ideal_gas_mixture_with_identity_change(oracle):
    ff = synthetic_forcefield(charges=False)
    ff.cutoff_molecule_vdw = 1e-3
    L = 30.0
    targets = (2.0, 5.0)
    comps = [co2_component(), n2_component()]
    fug = [t / (BETA * L ** 3) for t in targets]
    means = []
    for seed in range(6):
        r, _, _, _ = oracle.mixture_run(ff, np.diag([L, L, L]), comps, BETA, fug, np.zeros((0, 3, 3)),
                                        np.zeros(0, dtype=np.int32), 20000, seed=seed + 1, use_ewald=False)
        assert r["accepted"][4] > 0
        means.append([s / r["samples"] for s in r["sum_n"][:2]])
    means = np.array(means)
    for c, t in enumerate(targets):
        se = means[:, c].std(ddof=1) / math.sqrt(len(means))
        assert abs(means[:, c].mean() - t) < 4 * se + 0.03 * t, (c, means[:, c].mean(), t, se)


def test_framework_mixture_drift(oracle):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=6)
    for pa in ff.pseudo_atoms[:2]:
        pa.charge = 0.0
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (21, 21, 14)
    grids = [None] * (ff.n_types + 1)
    for name in ("C_co2", "O_co2", "N_n2"):
        grids[ff.index(name)] = oracle.make_grid(0, ff, ucell, ufw, ff.index(name), 12.0, dims)
    grids[ff.n_types] = oracle.make_grid(1, ff, ucell, ufw, 0, 12.0, dims)
    s_fw = oracle.ewald_rigid(ff, scell, sfw)
    comps = [co2_component(), n2_component()]
    r, xyz, comp, _ = oracle.mixture_run(ff, scell, comps, BETA, [fugacity_of(1e6), fugacity_of(1e6)],
                                         np.zeros((0, 3, 3)), np.zeros(0, dtype=np.int32), 3000, seed=3, grids=grids,
                                         grid_dims=dims, grid_cell=ucell, s_framework=s_fw)
    assert sum(r["n_molecules"]) == len(comp) > 0
    assert abs(r["running_energy"] - r["recomputed_energy"]) < 1e-8 * max(1.0, abs(r["recomputed_energy"]))
    # restart from the final configuration: the recomputed energy is the same
    r2, _, _, _ = oracle.mixture_run(ff, scell, comps, BETA, [fugacity_of(1e6), fugacity_of(1e6)], xyz, comp, 0,
                                     seed=4, grids=grids, grid_dims=dims, grid_cell=ucell, s_framework=s_fw)
    assert abs(r2["recomputed_energy"] - r["recomputed_energy"]) < 1e-9 * max(1.0, abs(r["recomputed_energy"]))

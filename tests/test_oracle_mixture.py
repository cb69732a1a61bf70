"""The CPU oracle of the mixture GCMC with identity change (oracle/mixture.cpp).

* Ideal-gas mixture (no framework, no intermolecular pairs, no Ewald): with translation, rotation, CBMC swap and
  identity change, <N_c> = beta f_c V for every component (the identity-change acceptance rule of
  mc_moves/component/identity_change.cpp:229-240 conserves the grand-canonical distribution).
* A small mixture in the synthetic framework (CO2 / N2 charged, Ewald on; framework charges off and on): the running
  energy equals the energy recomputed from scratch. N2's massless charge site has no grid and sees the framework atoms
  explicitly (interactions_framework_molecule.cpp, non-grid branch): with framework charges that term is nonzero.
"""

import math

import numpy as np
import pytest

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


@pytest.mark.parametrize("framework_charges", [False, True])
def test_framework_mixture_drift(oracle, framework_charges):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=6)
    if not framework_charges:
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
                                         grid_dims=dims, grid_cell=ucell, s_framework=s_fw, framework=sfw)
    assert sum(r["n_molecules"]) == len(comp) > 0
    assert abs(r["running_energy"] - r["recomputed_energy"]) < 1e-8 * max(1.0, abs(r["recomputed_energy"]))
    # restart from the final configuration: the recomputed energy is the same
    r2, _, _, _ = oracle.mixture_run(ff, scell, comps, BETA, [fugacity_of(1e6), fugacity_of(1e6)], xyz, comp, 0,
                                     seed=4, grids=grids, grid_dims=dims, grid_cell=ucell, s_framework=s_fw,
                                     framework=sfw)
    assert abs(r2["recomputed_energy"] - r["recomputed_energy"]) < 1e-9 * max(1.0, abs(r["recomputed_energy"]))
    # without the framework atoms the grid-less N_com sites lose their (charged-framework) Coulomb term
    assert (comp == 1).any()
    r3, _, _, _ = oracle.mixture_run(ff, scell, comps, BETA, [fugacity_of(1e6), fugacity_of(1e6)], xyz, comp, 0,
                                     seed=4, grids=grids, grid_dims=dims, grid_cell=ucell, s_framework=s_fw)
    if framework_charges:
        assert abs(r3["recomputed_energy"] - r["recomputed_energy"]) > 1.0
    else:
        assert r3["recomputed_energy"] == pytest.approx(r["recomputed_energy"], rel=1e-12, abs=1e-9)


def test_split_molecules_are_kept_whole(oracle):
    """Molecules handed in wrapped atom by atom (split across the box faces) are made whole by the minimum image before
    any move: rotations about the centre of mass keep the rigid geometry and the energy bookkeeping exact."""
    from raspa3_b200.mixture import random_mixture

    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=6)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (21, 21, 14)
    grids = [None] * (ff.n_types + 1)
    for name in ("C_co2", "O_co2", "N_n2"):
        grids[ff.index(name)] = oracle.make_grid(0, ff, ucell, ufw, ff.index(name), 12.0, dims)
    grids[ff.n_types] = oracle.make_grid(1, ff, ucell, ufw, 0, 12.0, dims)
    s_fw = oracle.ewald_rigid(ff, scell, sfw)
    comps = [co2_component(), n2_component()]
    xyz, comp = random_mixture(scell, sfw, comps, (20, 20), seed=3)
    L = np.diag(np.asarray(scell))
    split = xyz % L
    assert np.any(np.abs(split - xyz) > 1.0)  # at least one molecule is split
    r, out, comp_out, _ = oracle.mixture_run(ff, scell, comps, BETA, [fugacity_of(1e5), fugacity_of(1e5)], split, comp,
                                             3000, seed=5, grids=grids, grid_dims=dims, grid_cell=ucell,
                                             s_framework=s_fw, framework=sfw, probabilities=(0.2, 1.0, 0.0, 0.0))
    assert r["accepted"][1] > 100
    assert abs(r["running_energy"] - r["recomputed_energy"]) < 1e-8 * max(1.0, abs(r["recomputed_energy"]))
    for m, c in enumerate(comp_out):
        d_out = np.linalg.norm(out[m][:, None] - out[m][None], axis=-1)
        d_ref = np.linalg.norm(comps[c].offsets[:, None] - comps[c].offsets[None], axis=-1)
        assert np.allclose(d_out, d_ref, atol=1e-9)

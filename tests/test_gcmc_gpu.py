"""Device-resident GCMC (rg_gcmc) through the C-ABI: exact ideal-gas statistics, energy drift against an oracle
recomputation, and loading parity with the CPU oracle's GCMC (same moves, independent random streams)."""

import numpy as np

from chain_statistics import assert_agree
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, methane_component
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def empty_framework():
    return make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))


def chain_means(res):
    m = np.array([r["sum_n"] / r["samples"] for r in res])
    return m.mean(), m.std(ddof=1) / np.sqrt(len(m))


def loadings(res):
    return [r["sum_n"] / r["samples"] for r in res]


def test_ideal_gas_poisson(ctx):
    ff = synthetic_forcefield(charges=False)
    for p in ff.pseudo_atoms:
        p.epsilon_k = 0.0
    ff.__post_init__()
    cell = np.diag([30.0, 30.0, 30.0])
    beta, f = beta_of(300.0), fugacity_of(2e5)
    expected = beta * f * 27000.0
    sysg = native.System(ctx, ff, cell, empty_framework())
    g = native.Gcmc(sysg, None, co2_component(), beta, f, n_chains=256, seed=7)
    g.run(2000, record=False)
    g.run(8000, record=True)
    res = g.results()
    var = np.mean([r["sum_n2"] / r["samples"] - (r["sum_n"] / r["samples"]) ** 2 for r in res])
    assert_agree(loadings(res), expected=expected, label="ideal-gas <N> = beta f V")
    assert abs(var - expected) < 0.1 * expected
    assert all(abs(r["energy"]) < 1e-12 for r in res)


def co2_fluid(ctx, chains, seed):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=6)
    cell = np.diag([26.0, 26.0, 26.0])
    sysg = native.System(ctx, ff, cell, empty_framework())
    ew = native.Ewald(ctx, ff, cell)
    ew.set_framework(empty_framework())
    g = native.Gcmc(sysg, ew, co2_component(), beta_of(300.0), fugacity_of(4e6), n_chains=chains, seed=seed)
    return ff, cell, sysg, ew, g


def recompute(oracle, ff, cell, comp, xyz, grids=None, dims=None, ucell=None, s_fw=None):
    """Total energy of a configuration from scratch with the oracle (grids + pairs + Ewald)."""
    n_mol = len(xyz) // comp.n_atoms
    types = np.tile(comp.types(ff), n_mol).astype(np.uint16)
    q = np.tile(comp.charges(ff), n_mol)
    mids = np.repeat(np.arange(n_mol), comp.n_atoms)
    atoms = make_atoms(xyz, types, q, molecule_ids=mids)
    e = 0.0
    for m in range(n_mol):
        mol = atoms[m * comp.n_atoms:(m + 1) * comp.n_atoms]
        ok, ef = oracle.cbmc_framework_molecule(ff, cell, atoms[:0], mol, ff.cutoff_framework_vdw, ff.cutoff_coulomb,
                                                grids=grids, grid_dims=dims, grid_cell=ucell)
        e += ef["framework_molecule_vdw"] + ef["framework_molecule_charge"]
        ok, em = oracle.cbmc_intermolecular(ff, cell, atoms[(m + 1) * comp.n_atoms:], mol, ff.cutoff_molecule_vdw,
                                            ff.cutoff_coulomb)
        e += em["molecule_molecule_vdw"] + em["molecule_molecule_charge"]
    if ff.use_charge and n_mol:
        ee, _ = oracle.ewald_fourier_energy(ff, cell, atoms, [comp.n_atoms] * n_mol, s_rigid=s_fw)
        e += ee["ewald_fourier"] + ee["ewald_self"] + ee["ewald_exclusion"]
    return e


def test_co2_fluid_drift_and_parity_with_oracle(ctx, oracle):
    ff, cell, sysg, ew, g = co2_fluid(ctx, chains=128, seed=11)
    g.run(3000, record=False)
    g.run(12000, record=True)
    res = g.results()
    comp = co2_component()
    for c in range(4):
        xyz = g.positions(c)
        e = recompute(oracle, ff, cell, comp, xyz)
        assert abs(e - res[c]["energy"]) <= 1e-6 * max(1.0, abs(e)), (c, e, res[c]["energy"])
    m_gpu, err_gpu = chain_means(res)
    ref, _ = oracle.gcmc_run(ff, cell, comp, beta_of(300.0), fugacity_of(4e6), n_chains=16, steps=12000,
                             equilibration=3000, threads=0, seed=5)
    assert m_gpu > 2.0
    assert_agree(loadings(res), loadings(ref), label="CO2 fluid loading, device vs oracle")
    acc = np.sum([r["accepted"] for r in res], axis=0)
    assert np.all(acc > 0), acc


@pytest.fixture(scope="module")
def framework_co2(ctx, oracle):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (41, 41, 28)
    grids = [None] * (ff.n_types + 1)
    sysg = native.System(ctx, ff, scell, sfw)
    for idx, gt in ((ff.index("C_co2"), 0), (ff.index("O_co2"), 0), (ff.n_types, 1)):
        out, _ = ctx.grid_build(gt, ff, ucell, ufw, idx if gt == 0 else 0, 12.0, dims, native.PRECISION_FP64)
        grids[idx] = out
        sysg.set_grid(idx, ucell, dims, out)
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    s_fw = oracle.ewald_rigid(ff, scell, sfw)
    return dict(ff=ff, ucell=ucell, scell=scell, sfw=sfw, dims=dims, grids=grids, sys=sysg, ew=ew, s_fw=s_fw)


def test_framework_co2_drift(ctx, oracle, framework_co2):
    """The charged synthetic system (charged framework in a 2x2x3 box, grids, framework structure factor) at 1e5 Pa:
    every chain's running energy equals the oracle's recomputation of its final configuration."""
    c = framework_co2
    comp = co2_component()
    g = native.Gcmc(c["sys"], c["ew"], comp, beta_of(300.0), fugacity_of(1e5), n_chains=64, seed=3)
    g.run(4000, record=True)
    res = g.results()
    assert np.mean([r["n_molecules"] for r in res]) > 1
    for ch in range(3):
        xyz = g.positions(ch)
        e = recompute(oracle, c["ff"], c["scell"], comp, xyz, grids=c["grids"], dims=c["dims"], ucell=c["ucell"],
                      s_fw=c["s_fw"])
        assert abs(e - res[ch]["energy"]) <= 1e-6 * max(1.0, abs(e)), (ch, e, res[ch]["energy"])


def test_framework_co2_henry_regime_parity(ctx, oracle, framework_co2):
    """Low pressure (2 Pa): loading from the device chains vs the CPU oracle's chains."""
    c = framework_co2
    comp = co2_component()
    P = 2.0
    g = native.Gcmc(c["sys"], c["ew"], comp, beta_of(300.0), fugacity_of(P), n_chains=256, seed=9)
    g.run(2000, record=False)
    g.run(20000, record=True)
    res = g.results()
    m_gpu, err_gpu = chain_means(res)
    ref, _ = oracle.gcmc_run(c["ff"], c["scell"], comp, beta_of(300.0), fugacity_of(P), n_chains=16, steps=20000,
                             equilibration=2000, grids=c["grids"], grid_dims=c["dims"], grid_cell=c["ucell"],
                             s_framework=c["s_fw"], threads=0, seed=13)
    assert m_gpu > 0.05
    assert_agree(loadings(res), loadings(ref), label="framework CO2 loading at 2 Pa, device vs oracle")

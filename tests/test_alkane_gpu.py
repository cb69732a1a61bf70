"""Batched flexible-chain CBMC on the device (rg_alkane_*) against the FP64 CPU oracle and exact results.

Trial energies: FP32 pair terms from exact fixed-point displacements with FP64 reductions, checked per bead against
the FP64 oracle: |dE| <= 1e-6 * S + 1e-9 where S = sum over the bead's pairs of |e_pair| (the scale the FP32 rounding
of each pair term is relative to; for a bead in an attractive well S ~ |E|).
Sampling: the device draws the base conformation exactly and the oracle runs the reference's internal Monte Carlo,
so chains are compared in distribution and through exact results (butane's ideal-gas Rosenbluth weight by
quadrature, the ideal gas <N> = beta f V), and framework loadings are compared with the oracle's within statistical
error.
"""

import math

import numpy as np

from chain_statistics import assert_agree
import pytest

from raspa3_b200 import native
from raspa3_b200.alkane import AlkaneChain, AlkaneSystem, alkane_forcefield, alkane_batch_systems, replicate_for_cutoff
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, fugacity_of
from raspa3_b200.synthetic import synthetic_framework
from test_oracle_alkane import bend_exact_moments, butane_exact

pytestmark = pytest.mark.gpu
BETA = beta_of(300.0)


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def small_framework_system(ff, chain, w_ig, pressure=1e5, max_molecules=48, seed=42):
    """A 25 Angstrom cubic synthetic cell at 0.025 atoms per cubic Angstrom (130 T + 260 O): open enough for chains,
    wide enough for the minimum image of the 12 Angstrom cutoff without replication."""
    cell, atoms = synthetic_framework(ff, (25.0, 25.0, 25.0), n_t=130, seed=seed)
    scell, satoms, _ = replicate_for_cutoff(cell, atoms)
    return AlkaneSystem(cell=scell, framework=satoms, chain=chain, beta=BETA, fugacity=fugacity_of(pressure),
                        w_ig=w_ig, max_molecules=max_molecules)


def trans_chains(n_chains, nb, cell, rng, bond=1.54, theta_deg=114.0):
    """All-trans zig-zag chains at random positions and orientations: [n_chains, nb, 3]."""
    h = math.radians(theta_deg) / 2.0
    k = np.arange(nb)
    body = np.stack([k * bond * math.sin(h), (k % 2) * bond * math.cos(h), np.zeros(nb)], 1)
    body -= body.mean(0)
    out = []
    for _ in range(n_chains):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        out.append(body @ q.T + rng.random(3) @ np.asarray(cell))
    return np.array(out)


def pair_abs_sum(ff, q, xyz_mol, bead, t):
    """sum |e_pair| of one bead (FP64, numpy) over framework and molecule partners within the cutoffs."""
    cell = np.asarray(q.cell)
    inv = np.linalg.inv(cell)
    s = 0.0
    parts = [(np.stack([q.framework["x"], q.framework["y"], q.framework["z"]], 1), q.framework["type"],
              ff.cutoff_framework_vdw)]
    if len(xyz_mol):
        types = np.tile(q.chain.types(ff), len(xyz_mol))
        parts.append((xyz_mol.reshape(-1, 3), types, ff.cutoff_molecule_vdw))
    for pos, types, rc in parts:
        d = pos - bead
        f = d @ inv
        f -= np.rint(f)
        d = f @ cell
        rr = np.einsum("ij,ij->i", d, d)
        m = rr < rc * rc
        for tp in np.unique(types[m]):
            k = int(tp) * ff.n_types + t
            if not ff.lj.reshape(-1)[k]:
                continue
            eps, sig = ff.epsilon.reshape(-1)[k], ff.sigma.reshape(-1)[k]
            x = (sig * sig / rr[m & (types == tp)]) ** 3
            s += float(np.sum(np.abs(4 * eps * x * (x - 1) - ff.shift.reshape(-1)[k])))
    return s


def test_bead_energies_match_oracle(ctx, oracle):
    ff = alkane_forcefield()
    ch = AlkaneChain(6)
    q = small_framework_system(ff, ch, 1.0)
    rng = np.random.default_rng(5)
    xyz = trans_chains(6, ch.n_beads, q.cell, rng)
    a = native.Alkane(ctx, ff, [q], seed=3)
    a.set_positions(0, xyz)
    cell = np.asarray(q.cell)
    beads = rng.random((16, 3)) @ cell
    # include beads sitting on existing chains' sites and near them (molecule-molecule terms), and skip handling
    beads[:4] = xyz[0, :4] + rng.normal(scale=0.8, size=(4, 3))
    types = np.array([ff.index("CH2")] * 8 + [ff.index("CH3")] * 8, dtype=np.int32)
    for skip in (-1, 0):
        fw, mm, ov = a.bead_energies(0, beads, types, skip=skip)
        rfw, rmm, rov = oracle.alkane_bead_energies(ff, q, xyz, beads, types, skip=skip)
        assert np.array_equal(ov, rov)
        for b in range(16):
            if ov[b]:
                continue
            sc = pair_abs_sum(ff, q, np.delete(xyz, skip, 0) if skip >= 0 else xyz, beads[b], int(types[b]))
            err = abs(fw[b] + mm[b] - rfw[b] - rmm[b])
            assert err <= 1e-6 * sc + 1e-9, (b, fw[b], rfw[b], mm[b], rmm[b], sc)
            assert abs(mm[b] - rmm[b]) <= 1e-6 * sc + 1e-9
    a.close()


def test_butane_vacuum_growth_exact(ctx):
    ff = alkane_forcefield()
    ch = AlkaneChain(4)
    mean, w, th, cp = native.alkane_grow_vacuum(ctx, ff, ch, BETA, 200000, seed=7, details=True)
    w_ig, cos_avg = butane_exact(ch, ff)
    se = w.std(ddof=1) / math.sqrt(len(w))
    assert abs(mean - w_ig) < 4 * se, (mean, w_ig, se)
    cw = float(np.sum(w * cp[:, 0]) / np.sum(w))
    assert abs(cw - cos_avg) < 0.005, (cw, cos_avg)
    m1, sd = bend_exact_moments(ch, ff)
    x = th.reshape(-1)
    assert abs(x.mean() - m1) < 4 * sd / math.sqrt(len(x)), (x.mean(), m1)
    assert abs(x.std() - sd) < 0.01 * sd


def test_vacuum_growth_matches_oracle(ctx, oracle):
    """Octane in vacuum (1-5 and longer intra-molecular pairs enter the weights): <W>, the W-weighted torsion
    average and the bend-angle moments agree between the device and the oracle's internal Monte Carlo."""
    ff = alkane_forcefield()
    ch = AlkaneChain(8)
    mean, w, th, cp = native.alkane_grow_vacuum(ctx, ff, ch, BETA, 200000, seed=8, details=True)
    wo, tho, cpo = oracle.alkane_grow_vacuum(ff, ch, BETA, 40000, seed=8)
    se = math.hypot(w.std(ddof=1) / math.sqrt(len(w)), wo.std(ddof=1) / math.sqrt(len(wo)))
    assert abs(mean - wo.mean()) < 4 * se, (mean, wo.mean(), se)
    for j in range(cp.shape[1]):
        a = np.sum(w * cp[:, j]) / np.sum(w)
        b = np.sum(wo * cpo[:, j]) / np.sum(wo)
        assert abs(a - b) < 0.03, (j, a, b)
    assert abs(th.mean() - tho.mean()) < 1e-3
    assert abs(th.std() - tho.std()) < 0.02 * tho.std()


def test_ideal_gas_loading(ctx):
    ff = alkane_forcefield()
    ff.cutoff_molecule_vdw = 1e-3
    ch = AlkaneChain(6)
    w_ig, w, _, _ = native.alkane_grow_vacuum(ctx, ff, ch, BETA, 400000, seed=9, details=True)
    w_ig_rel_err = w.std(ddof=1) / math.sqrt(len(w)) / w_ig  # the loading scales with 1 / W_IG
    L, target = 30.0, 3.0
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    systems = [AlkaneSystem(cell=np.diag([L, L, L]), framework=empty, chain=ch, beta=BETA,
                            fugacity=target / (BETA * L ** 3), w_ig=w_ig, max_molecules=64) for _ in range(256)]
    a = native.Alkane(ctx, ff, systems, seed=21)
    a.run(1000, record=False)
    a.run(6000, record=True)
    res = a.results()
    means = np.array([r["sum_n"] / r["samples"] for r in res])
    # the chains' standard error and the propagated error of the estimated W_IG, no slack
    se = math.hypot(means.std(ddof=1) / math.sqrt(len(means)), target * w_ig_rel_err)
    z = (means.mean() - target) / se
    print(f"ideal-gas alkane loading {means.mean():.5f} vs {target} (se {se:.2g}): z = {z:+.2f}")
    assert abs(z) < 4, (means.mean(), se, z)
    a.close()


@pytest.mark.parametrize("plan", [(1, 1, 128), (2, 2, 256), (4, 2, 128), (1, 1, 512)])
def test_loading_matches_oracle_and_no_drift(ctx, oracle, plan):
    """Pentane at 1e5 Pa in the 25 Angstrom low-density cell: 128 device replicas vs 32 oracle replicas,
    under several launch plans (cluster sizes, threads), and the running energy against an FP64 recomputation of the
    final state."""
    ff = alkane_forcefield()
    ch = AlkaneChain(5)
    w_ig = native.alkane_grow_vacuum(ctx, ff, ch, BETA, 200000, seed=10)
    q = small_framework_system(ff, ch, w_ig, pressure=1e5)
    a = native.Alkane(ctx, ff, [q] * 128, seed=31)
    a.set_plan(cluster_big=plan[0], cluster_small=plan[1], threads=plan[2], split=64, moves_per_launch=50)
    a.run(1500, record=False)
    a.run(3000, record=True)
    res = a.results()
    gm = np.array([r["sum_n"] / r["samples"] for r in res])
    ores, _, _ = oracle.alkane_run(ff, [q] * 32, steps=3000, equilibration=1500, seed=6)
    om = np.array([r["sum_n"] / r["samples"] for r in ores])
    assert gm.mean() > 0.5
    assert_agree(gm, om, label=f"pentane loading, device plan {plan} vs oracle")
    for s in range(0, 128, 37):
        x = a.positions(s)
        e = oracle.alkane_energy(ff, q, x)
        tot = sum(e)
        assert abs(res[s]["energy"] - tot) < 1e-5 * max(1.0, abs(tot)) + 1e-4, (s, res[s]["energy"], tot)
    a.close()


def test_batched_uneven_systems_autotune(ctx, oracle):
    """Eight uneven batched-alkane systems (cells, chain lengths, trial counts): the autotuner picks a plan, the
    run completes with every system's running energy equal to an FP64 recomputation of its final state."""
    ff = alkane_forcefield()
    trials = [(10, 10), (8, 12), (16, 6), (10, 10), (4, 16), (12, 8), (10, 10), (6, 14)]
    systems = alkane_batch_systems(ff, n_systems=8, seed=77, trials=trials)
    for q in systems:
        q.w_ig = native.alkane_grow_vacuum(ctx, ff, q.chain, BETA, 50000, seed=3)
    a = native.Alkane(ctx, ff, systems, seed=41)
    plan = a.autotune(moves_per_candidate=4)
    assert plan["threads"] in (128, 256, 512) and plan["cluster_big"] in (1, 2, 4)
    a.run(600, record=True)
    res = a.results()
    assert sum(r["accepted"][2] for r in res) > 0
    for s, q in enumerate(systems):
        x = a.positions(s)
        assert len(x) == res[s]["n_molecules"]
        tot = sum(oracle.alkane_energy(ff, q, x))
        assert abs(res[s]["energy"] - tot) < 1e-5 * max(1.0, abs(tot)) + 1e-4, (s, res[s]["energy"], tot)
    a.close()

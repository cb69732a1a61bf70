"""The CPU oracle of flexible-chain CBMC (oracle/alkane.cpp) against exact results.

* Butane grown in vacuum: every direction and spin of a step has the same external energy, so the Rosenbluth weight
  of a chain is the torsion weight of its last step and <W> = <exp(-beta U_tors(phi))> over a uniform phi (the
  ideal-gas Rosenbluth weight, by quadrature). The W-weighted torsion average is the Boltzmann average.
* The bend angles of grown chains follow p(theta) ~ sin(theta) exp(-beta U_bend(theta)), the stationary distribution
  of the reference's internal bond/bend Monte Carlo (cbmc/operators.cpp:203-447).
* Ideal gas (no framework, no intermolecular pairs) with W_IG = <W>: <N> = beta f V.
* A framework system: the running energy equals the energy recomputed from the final positions.
"""

import math

import numpy as np
import pytest

from raspa3_b200.alkane import AlkaneChain, AlkaneSystem, alkane_forcefield, chain_struct, replicate_for_cutoff
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, fugacity_of
from raspa3_b200.synthetic import synthetic_framework

BETA = beta_of(300.0)


def torsion_energy(chain, ff, cos_phi):
    c = chain_struct(chain, ff)
    p = list(c.torsion)
    return p[0] + (1.0 + cos_phi) * (p[1] + p[3] - 2.0 * (cos_phi - 1.0) * (p[2] - 2.0 * p[3] * cos_phi))


def butane_exact(chain, ff):
    phi = np.linspace(-math.pi, math.pi, 200001)
    bf = np.exp(-BETA * torsion_energy(chain, ff, np.cos(phi)))
    w_ig = np.trapezoid(bf, phi) / (2 * math.pi)
    cos_avg = np.trapezoid(bf * np.cos(phi), phi) / np.trapezoid(bf, phi)
    return w_ig, cos_avg


def bend_exact_moments(chain, ff):
    c = chain_struct(chain, ff)
    th = np.linspace(1e-6, math.pi - 1e-6, 200001)
    p = np.sin(th) * np.exp(-BETA * 0.5 * c.bend_k * (th - c.bend_theta0) ** 2)
    z = np.trapezoid(p, th)
    m1 = np.trapezoid(p * th, th) / z
    m2 = np.trapezoid(p * th * th, th) / z
    return m1, math.sqrt(m2 - m1 * m1)


def test_butane_vacuum_weight_and_torsions(oracle):
    ff = alkane_forcefield()
    ch = AlkaneChain(4)
    w, th, cp = oracle.alkane_grow_vacuum(ff, ch, BETA, 40000, seed=11)
    w_ig, cos_avg = butane_exact(ch, ff)
    se = w.std(ddof=1) / math.sqrt(len(w))
    assert abs(w.mean() - w_ig) < 4 * se, (w.mean(), w_ig, se)
    cw = float(np.sum(w * cp[:, 0]) / np.sum(w))
    assert abs(cw - cos_avg) < 0.01, (cw, cos_avg)


def test_bend_angle_distribution(oracle):
    ff = alkane_forcefield()
    ch = AlkaneChain(5)
    _, th, _ = oracle.alkane_grow_vacuum(ff, ch, BETA, 20000, seed=12)
    m1, sd = bend_exact_moments(ch, ff)
    x = th.reshape(-1)
    assert abs(x.mean() - m1) < 4 * sd / math.sqrt(len(x)) + 1e-4, (x.mean(), m1)
    assert abs(x.std() - sd) < 0.02 * sd, (x.std(), sd)


def empty_system(chain, ff, L, n_expected, w_ig):
    V = L ** 3
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    return AlkaneSystem(cell=np.diag([L, L, L]), framework=empty, chain=chain, beta=BETA,
                        fugacity=n_expected / (BETA * V), w_ig=w_ig, max_molecules=64)


def test_ideal_gas_loading(oracle):
    ff = alkane_forcefield()
    ff.cutoff_molecule_vdw = 1e-3  # no intermolecular pairs
    ch = AlkaneChain(6)
    w, _, _ = oracle.alkane_grow_vacuum(ff, ch, BETA, 40000, seed=13)
    systems = [empty_system(ch, ff, 30.0, 3.0, float(w.mean())) for _ in range(32)]
    res, _, _ = oracle.alkane_run(ff, systems, steps=4000, equilibration=500, seed=4)
    means = np.array([r["sum_n"] / r["samples"] for r in res])
    se = means.std(ddof=1) / math.sqrt(len(means))
    # the W_IG estimate itself carries a relative error se_w / <W>
    rel_w = w.std(ddof=1) / math.sqrt(len(w)) / w.mean()
    assert abs(means.mean() - 3.0) < 4 * math.hypot(se, 3.0 * rel_w), (means.mean(), se)


def test_framework_drift(oracle):
    ff = alkane_forcefield()
    cell, atoms = synthetic_framework(ff, (20.0, 19.9, 13.4), n_t=96, seed=42)
    scell, satoms, _ = replicate_for_cutoff(cell, atoms)
    ch = AlkaneChain(5)
    w, _, _ = oracle.alkane_grow_vacuum(ff, ch, BETA, 20000, seed=14)
    q = AlkaneSystem(cell=scell, framework=satoms, chain=ch, beta=BETA, fugacity=fugacity_of(1e5),
                     w_ig=float(w.mean()), max_molecules=64)
    res, pos, _ = oracle.alkane_run(ff, [q, q], steps=600, equilibration=0, seed=5)
    for r, x in zip(res, pos):
        assert r["n_molecules"] == len(x)
        assert abs(r["running_energy"] - r["recomputed_energy"]) < 1e-8 * max(1.0, abs(r["recomputed_energy"]))
        e = oracle.alkane_energy(ff, q, x)
        assert abs(sum(e) - r["recomputed_energy"]) < 1e-9 * max(1.0, abs(sum(e)))

"""Learned first-bead proposal: hand-written MLP kernels vs the FP64 numpy oracle, training, exact normalisation,
and the GCMC ensemble it samples (unchanged by construction, checked here)."""

import numpy as np

from chain_statistics import assert_agree
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


def mlp_oracle():
    import importlib

    return importlib.import_module("oracle.mlp")


def test_forward_and_gradient_match_fp64_oracle(ctx, torch):
    mo = mlp_oracle()
    m = native.Mlp(ctx, seed=5)
    theta = m.params().astype(np.float64)
    assert len(theta) == mo.N_PARAMS == 10433
    rng = np.random.default_rng(0)
    n = 1000
    s = rng.random((n, 3)).astype(np.float32)
    t = (rng.normal(size=n) * 3.0).astype(np.float32)
    ds = torch.from_numpy(s).cuda()
    dt = torch.from_numpy(t).cuda()
    out = torch.empty(n, dtype=torch.float32, device="cuda")
    m.evaluate(ds.data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    f_ref = mo.forward(theta, s.astype(np.float64))
    f_gpu = out.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(f_gpu - f_ref)) < 1e-4 * max(1.0, np.sqrt(np.mean(f_ref ** 2)))
    loss, grad = m.loss_and_gradient(ds.data_ptr(), dt.data_ptr(), n)
    loss_ref, grad_ref = mo.loss_and_grad(theta, s.astype(np.float64), t.astype(np.float64))
    assert abs(loss - loss_ref) < 1e-4 * loss_ref
    rel = np.linalg.norm(grad.astype(np.float64) - grad_ref) / np.linalg.norm(grad_ref)
    assert rel < 1e-4, rel
    # every block of the parameter vector, separately (W1, b1, W2, b2, w3, b3)
    cuts = np.cumsum([0, 64 * 96, 64, 64 * 64, 64, 64, 1])
    for a, b in zip(cuts[:-1], cuts[1:]):
        den = np.linalg.norm(grad_ref[a:b]) + 1e-30
        assert np.linalg.norm(grad[a:b] - grad_ref[a:b]) / den < 1e-3, (a, b)


def test_training_reduces_loss_on_smooth_target(ctx, torch):
    m = native.Mlp(ctx, seed=2)
    rng = np.random.default_rng(1)
    n = 1 << 16
    s = rng.random((n, 3)).astype(np.float32)
    t = (3.0 * np.cos(2 * np.pi * s[:, 0]) * np.sin(2 * np.pi * s[:, 1]) + np.cos(4 * np.pi * s[:, 2])).astype(
        np.float32)
    ds, dt = torch.from_numpy(s).cuda(), torch.from_numpy(t).cuda()
    l0, _ = m.loss_and_gradient(ds.data_ptr(), dt.data_ptr(), 4096)
    l1 = m.train(ds.data_ptr(), dt.data_ptr(), n, steps=1500, batch=2048, lr=2e-3)
    assert l1 < 0.02 * l0, (l0, l1)


def test_proposal_is_normalised(ctx):
    m = native.Mlp(ctx, seed=3)
    G = 16
    p = native.Proposal(m, cells_per_axis=G, eps_uniform=0.1)
    c = (np.stack(np.meshgrid(np.arange(G), np.arange(G), np.arange(G), indexing="ij"), -1).reshape(-1, 3) + 0.5) / G
    q = p.density(c)
    assert abs(q.mean() - 1.0) < 1e-12
    assert q.min() >= 0.1 - 1e-12


def empty_framework():
    return make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))


def test_ideal_gas_unchanged_by_a_biased_proposal(ctx, torch):
    """With interactions off, <N> = beta f V for any proposal: a strongly non-uniform one (an MLP trained on a sharp
    synthetic target) must still sample the Poisson distribution exactly (detailed balance of the biased CBMC)."""
    ff = synthetic_forcefield(charges=False)
    for pa in ff.pseudo_atoms:
        pa.epsilon_k = 0.0
    ff.__post_init__()
    ucell = np.diag([15.0, 15.0, 15.0])
    cell = np.diag([30.0, 30.0, 30.0])
    m = native.Mlp(ctx, seed=4)
    rng = np.random.default_rng(2)
    n = 1 << 15
    s = rng.random((n, 3)).astype(np.float32)
    t = (-8.0 * ((s - 0.3) ** 2).sum(1) * 10).astype(np.float32)
    ds, dt = torch.from_numpy(s).cuda(), torch.from_numpy(t).cuda()
    m.train(ds.data_ptr(), dt.data_ptr(), n, steps=600, batch=2048, lr=2e-3)
    prop = native.Proposal(m, cells_per_axis=32, eps_uniform=0.05)
    beta, f = beta_of(300.0), fugacity_of(2e5)
    expected = beta * f * 27000.0
    sysg = native.System(ctx, ff, cell, empty_framework())
    g = native.Gcmc(sysg, None, co2_component(), beta, f, n_chains=256, seed=17)
    g.set_proposal(prop, ucell)
    g.run(2000, record=False)
    g.run(8000, record=True)
    res = g.results()
    assert_agree([r["sum_n"] / r["samples"] for r in res], expected=expected,
                 label="ideal-gas <N> under a non-uniform proposal")


def test_learned_proposal_same_loading_higher_swap_acceptance(ctx, torch):
    """CO2 (charged, Ewald) in the synthetic framework with the framework charges switched off (with them the binding
    wells of ~-1e4 K make every sampler non-ergodic), 1e6 Pa: the proposal is trained on the C atom's grid Boltzmann
    factors. Learned and uniform chains agree on the loading within error; the learned one accepts more swaps."""
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    for pa in ff.pseudo_atoms[:2]:
        pa.charge = 0.0
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (67, 67, 45)
    sysg = native.System(ctx, ff, scell, sfw)
    keep = []
    for idx, gt in ((ff.index("C_co2"), 0), (ff.index("O_co2"), 0), (ff.n_types, 1)):
        buf = torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
        ctx.grid_build(gt, ff, ucell, ufw, idx if gt == 0 else 0, 12.0, dims, native.PRECISION_FP32C,
                       out_device=buf.data_ptr(), host=False)
        sysg.set_grid(idx, ucell, dims, buf.data_ptr(), on_device=True)
        keep.append(buf)
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    beta = beta_of(300.0)
    n = 1 << 20
    ds = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    dt = torch.empty(n, dtype=torch.float32, device="cuda")
    comp = co2_component()
    c_atom = comp.starting_bead
    native.sample_targets(sysg, int(comp.types(ff)[c_atom]), float(comp.charges(ff)[c_atom]), beta, -15.0, ucell, n, 9,
                          ds.data_ptr(), dt.data_ptr())
    m = native.Mlp(ctx, seed=1)
    m.train(ds.data_ptr(), dt.data_ptr(), n, steps=2000, batch=4096, lr=2e-3)
    prop = native.Proposal(m, cells_per_axis=48, eps_uniform=0.05)
    runs = {}
    for name, use in (("uniform", False), ("learned", True)):
        g = native.Gcmc(sysg, ew, comp, beta, fugacity_of(1e6), n_chains=512, seed=21 if use else 22)
        if use:
            g.set_proposal(prop, ucell)
        g.run(4000, record=False)
        g.run(12000, record=True)
        runs[name] = g.results()

    def summary(res):
        means = np.array([r["sum_n"] / r["samples"] for r in res])
        acc = np.sum([r["accepted"] for r in res], axis=0)
        att = np.sum([r["attempted"] for r in res], axis=0)
        return means.mean(), means.std(ddof=1) / np.sqrt(len(means)), (acc[2] + acc[3]) / max(1, att[2] + att[3])

    mu, eu, au = summary(runs["uniform"])
    ml, el, al = summary(runs["learned"])
    print("uniform", mu, eu, au, "learned", ml, el, al)
    assert mu > 0.5
    assert al > au
    # the learned proposal leaves the ensemble unchanged: loading and energy agree within their errors
    def per_chain(res, key):
        return [r[key] / r["samples"] for r in res]

    assert_agree(per_chain(runs["learned"], "sum_n"), per_chain(runs["uniform"], "sum_n"),
                 label="loading, learned vs uniform proposal")
    assert_agree(per_chain(runs["learned"], "sum_energy"), per_chain(runs["uniform"], "sum_energy"),
                 label="energy, learned vs uniform proposal")

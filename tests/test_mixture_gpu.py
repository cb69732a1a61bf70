"""One large mixture system on the whole GPU (rg_mixture_*) against exact results and the FP64 CPU oracle.

* Ideal-gas mixture with translation, rotation, CBMC swap and identity change: <N_c> = beta f_c V per component.
* CO2 + N2 in the synthetic framework (the adsorbates charged, Ewald on; framework charges off and on): the running
  energy and the structure factors after thousands of moves equal an FP64 recomputation of the final configuration,
  and the loading of each component agrees with independent oracle runs on the same grids. N2's massless charge site
  has no grid, so it sees the framework atoms explicitly (the reference's non-grid branch), on both sides.
* The large configuration (4 x 4 x 4 framework cells, 2,000 CO2 + 2,000 N2, kmax 12) runs without a barrier
  timeout and without drift.
"""

import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from chain_statistics import assert_agree
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, n2_component
from raspa3_b200.mixture import large_mixture, random_mixture, total_energy
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu
BETA = beta_of(300.0)
N_RUNS = 16  # independent runs per side in the loading comparison
RECORDED = 50000  # recorded moves per run after 3000 discarded equilibration moves


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def test_ideal_gas_mixture_with_identity_change(ctx):
    ff = synthetic_forcefield(charges=False)
    ff.cutoff_molecule_vdw = 1e-3
    L = 30.0
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    sysg = native.System(ctx, ff, np.diag([L, L, L]), empty)
    targets = (2.0, 5.0)
    comps = [co2_component(), n2_component()]
    means = []
    for seed in range(8):
        mx = native.Mixture(sysg, None, comps, BETA, [t / (BETA * L ** 3) for t in targets], np.zeros((0, 3, 3)),
                            np.zeros(0, dtype=np.int32), max_molecules=256, seed=seed + 1)
        mx.set_state(0.0)
        mx.run(2000, record=False)
        mx.run(20000, record=True)
        r = mx.results()
        assert r["status"] == 0 and r["accepted"][4] > 0
        means.append([s / r["samples"] for s in r["sum_n"][:2]])
        mx.close()
    means = np.array(means)
    for c, t in enumerate(targets):
        assert_agree(means[:, c], expected=t, label=f"ideal-gas mixture <N> of component {c}")


def framework_system(ctx, torch, kmax=6, framework_charges=False):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=kmax)
    if not framework_charges:
        for pa in ff.pseudo_atoms[:2]:
            pa.charge = 0.0
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (34, 34, 23)
    sysg = native.System(ctx, ff, scell, sfw)
    bufs, host = [], [None] * (ff.n_types + 1)
    for name, gt in (("C_co2", 0), ("O_co2", 0), ("N_n2", 0), (None, 1)):
        idx = ff.index(name) if name else ff.n_types
        buf = torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda")
        ctx.grid_build(gt, ff, ucell, ufw, idx if gt == 0 else 0, 12.0, dims, native.PRECISION_FP64,
                       out_device=buf.data_ptr(), host=False)
        sysg.set_grid(idx, ucell, dims, buf.data_ptr(), on_device=True)
        bufs.append(buf)
    # the builds ran on the context's own stream; torch's copies below run on torch's stream
    ctx.synchronize()
    for idx, buf in zip([ff.index("C_co2"), ff.index("O_co2"), ff.index("N_n2"), ff.n_types], bufs):
        host[idx] = buf.cpu().numpy()
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    return ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host


@pytest.mark.parametrize("framework_charges", [False, True])
def test_framework_mixture_drift_and_loading(ctx, torch, oracle, framework_charges):
    ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host = framework_system(ctx, torch,
                                                                               framework_charges=framework_charges)
    comps = [co2_component(), n2_component()]
    fug = [fugacity_of(1e6), fugacity_of(1e6)]
    runs = []
    for seed in range(N_RUNS):
        mx = native.Mixture(sysg, ew, comps, BETA, fug, np.zeros((0, 3, 3)), np.zeros(0, dtype=np.int32),
                            max_molecules=256, seed=seed + 11)
        mx.set_state(0.0, ew.structure_factors(2))
        mx.run(3000, record=False)
        mx.run(RECORDED, record=True)
        r = mx.results()
        assert r["status"] == 0
        runs.append([s / r["samples"] for s in r["sum_n"][:2]])
        if seed == 0:
            xyz, comp = mx.positions()
            assert len(comp) == sum(r["n_molecules"]) > 0
            e = total_energy(sysg, ew, ff, comps, xyz, comp)
            assert abs(r["energy"] - e) < 1e-5 * max(1.0, abs(e)), (r["energy"], e)
            sk = mx.structure_factors()
            ref = ew.structure_factors(0)
            assert np.max(np.abs(sk - ref)) < 1e-9 * max(1.0, np.max(np.abs(ref)))
        mx.close()
    gpu = np.array(runs)
    s_fw = ew.structure_factors(2)

    kw = dict(grids=host, grid_dims=dims, grid_cell=ucell, s_framework=s_fw, max_molecules=256, framework=sfw)

    def one(seed):
        # the same 3000 equilibration moves, discarded, then RECORDED from the equilibrated configuration
        _, xyz0, comp0, _ = oracle.mixture_run(ff, scell, comps, BETA, fug, np.zeros((0, 3, 3)),
                                               np.zeros(0, dtype=np.int32), 3000, seed=seed, **kw)
        r, _, _, _ = oracle.mixture_run(ff, scell, comps, BETA, fug, xyz0, comp0, RECORDED, seed=seed + 100, **kw)
        return r

    with ThreadPoolExecutor(N_RUNS) as pool:
        ores = list(pool.map(one, range(N_RUNS)))
    cpu = np.array([[s / r["samples"] for s in r["sum_n"][:2]] for r in ores])
    for c in range(2):
        assert_agree(gpu[:, c], cpu[:, c], label=f"mixture loading of component {c}, device vs oracle")


def test_split_molecules_are_kept_whole(ctx, torch):
    """Molecules handed in wrapped atom by atom (split across the box faces): rg_mixture_create makes them whole, so
    rotations keep the rigid geometry and the running energy equals the recomputed one."""
    ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host = framework_system(ctx, torch, framework_charges=True)
    comps = [co2_component(), n2_component()]
    xyz, comp = random_mixture(scell, sfw, comps, (20, 20), seed=3)
    split = xyz % np.diag(np.asarray(scell))
    assert np.any(np.abs(split - xyz) > 1.0)
    e0 = total_energy(sysg, ew, ff, comps, xyz, comp)
    sk0 = ew.structure_factors(0)
    mx = native.Mixture(sysg, ew, comps, BETA, [fugacity_of(1e5), fugacity_of(1e5)], split, comp, max_molecules=256,
                        seed=5, probabilities=(0.2, 1.0, 0.0, 0.0))
    mx.set_state(e0, sk0)
    mx.run(3000, record=True)
    r = mx.results()
    assert r["status"] == 0 and r["accepted"][1] > 100
    out, comp_out = mx.positions()
    for m, c in enumerate(comp_out):
        d_out = np.linalg.norm(out[m][:, None] - out[m][None], axis=-1)
        d_ref = np.linalg.norm(comps[c].offsets[:, None] - comps[c].offsets[None], axis=-1)
        assert np.allclose(d_out, d_ref, atol=1e-9)
    e = total_energy(sysg, ew, ff, comps, out, comp_out)
    assert abs(r["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (r["energy"], e)
    mx.close()


def test_large_mixture_runs_without_drift(ctx, torch):
    d = large_mixture(ctx, torch)
    ff, comps = d["ff"], d["components"]
    e0 = total_energy(d["system"], d["ewald"], ff, comps, d["xyz"], d["comp"])
    sk0 = d["ewald"].structure_factors(0)
    mx = native.Mixture(d["system"], d["ewald"], comps, BETA, [fugacity_of(1e5), fugacity_of(1e5)], d["xyz"],
                        d["comp"], max_molecules=6000, seed=7)
    info = mx.info()
    assert info["n_kvectors"] == 13 * 25 * 25 - 1  # the full half-box of kmax 12
    mx.set_state(e0, sk0)
    mx.run(2000, record=True)
    r = mx.results()
    assert r["status"] == 0
    assert sum(r["accepted"]) > 0
    xyz, comp = mx.positions()
    e = total_energy(d["system"], d["ewald"], ff, comps, xyz, comp)
    assert abs(r["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (r["energy"], e)
    mx.close()


@pytest.mark.parametrize("blocks,n_systems", [(4, 3), (2, 2)])
def test_large_mixtures_on_few_ctas_each(ctx, torch, blocks, n_systems):
    """The large mixture (12,000 sites, 8,124 k-vectors) with 2 or 4 CTAs per system (2,031 or 4,062 k-vectors per CTA: several tiles of the candidates'
    energy sums; at 2 CTAs most of the 6,000 sites per CTA come from L2 beyond the staged slice), several systems per
    launch: each system equals the same system run on its own, its running energy equals an FP64 recomputation of its
    final configuration, and its structure factors equal a recomputation."""
    d = large_mixture(ctx, torch)
    ff, comps = d["ff"], d["components"]
    e0 = total_energy(d["system"], d["ewald"], ff, comps, d["xyz"], d["comp"])
    sk0 = d["ewald"].structure_factors(0)

    def make(s):
        mx = native.Mixture(d["system"], d["ewald"], comps, BETA, [fugacity_of(1e5), fugacity_of(1e5)], d["xyz"],
                            d["comp"], max_molecules=6000, seed=11 + s, n_blocks=blocks)
        mx.set_state(e0, sk0)
        return mx

    batch = [make(s) for s in range(n_systems)]
    native.Mixture.run_many(batch, 400)
    alone = make(0)
    alone.run(400)
    assert batch[0].results() == alone.results()
    np.testing.assert_array_equal(batch[0].structure_factors(), alone.structure_factors())
    for mx in batch:
        r = mx.results()
        assert r["status"] == 0 and sum(r["accepted"]) > 0
        xyz, comp = mx.positions()
        e = total_energy(d["system"], d["ewald"], ff, comps, xyz, comp)  # leaves this configuration's S(k) behind
        assert abs(r["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (r["energy"], e)
        ref = d["ewald"].structure_factors(0)
        assert np.max(np.abs(mx.structure_factors() - ref)) < 1e-9 * max(1.0, np.max(np.abs(ref)))
    # the systems of one launch must share everything but their state
    other = native.Mixture(d["system"], d["ewald"], comps, BETA, [fugacity_of(2e5), fugacity_of(1e5)], d["xyz"],
                           d["comp"], max_molecules=6000, seed=99, n_blocks=blocks)
    with pytest.raises(native.RaspaGpuError):
        native.Mixture.run_many([batch[0], other], 1)
    for mx in batch + [alone, other]:
        mx.close()


def test_several_mixtures_in_one_launch_equal_separate_runs(ctx, torch):
    """rg_mixture_run_many: independent systems on disjoint CTA groups of one cooperative launch give exactly the
    results of the same systems run on their own (the same CTA count, seeds and moves), and each still matches an FP64
    recomputation of its final configuration."""
    ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host = framework_system(ctx, torch, framework_charges=True)
    comps = [co2_component(), n2_component()]
    fug = [fugacity_of(1e6), fugacity_of(1e6)]
    starts = [random_mixture(scell, sfw, comps, (6, 6), seed=40 + s) for s in range(3)]

    def make(s):
        xyz, comp = starts[s]
        e0 = total_energy(sysg, ew, ff, comps, xyz, comp)  # also leaves this configuration's S(k) in the Ewald state
        mx = native.Mixture(sysg, ew, comps, BETA, fug, xyz, comp, max_molecules=128, seed=70 + s, n_blocks=37)
        mx.set_state(e0, ew.structure_factors(0))
        return mx

    batch = [make(s) for s in range(3)]
    native.Mixture.run_many(batch, 1500)
    alone = []
    for s in range(3):
        mx = make(s)
        mx.run(1500)
        alone.append(mx)
    for b, a in zip(batch, alone):
        rb, ra = b.results(), a.results()
        assert rb["status"] == ra["status"] == 0
        assert rb == ra, (rb, ra)
        xb, cb = b.positions()
        xa, ca = a.positions()
        np.testing.assert_array_equal(xb, xa)
        np.testing.assert_array_equal(b.structure_factors(), a.structure_factors())
        e = total_energy(sysg, ew, ff, comps, xb, cb)
        assert abs(rb["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (rb["energy"], e)
    for m in batch + alone:
        m.close()
    with pytest.raises(native.RaspaGpuError):  # the systems' CTAs must fit on the GPU at once
        big = [native.Mixture(sysg, ew, comps, BETA, fug, starts[0][0], starts[0][1], max_molecules=128, seed=1,
                              n_blocks=100) for _ in range(2)]
        try:
            native.Mixture.run_many(big, 10)
        finally:
            for m in big:
                m.close()

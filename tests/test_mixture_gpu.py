"""One large mixture system on the whole GPU (rg_mixture_*) against exact results and the FP64 CPU oracle.

* Ideal-gas mixture with translation, rotation, CBMC swap and identity change: <N_c> = beta f_c V per component.
* CO2 + N2 in the synthetic framework (framework charges off, the adsorbates charged, Ewald on): the running energy and
  the structure factors after thousands of moves equal an FP64 recomputation of the final configuration, and the
  loading of each component agrees with independent oracle runs on the same grids.
* The large configuration (4 x 4 x 4 framework cells, 2,000 CO2 + 2,000 N2, kmax 12) runs without a barrier
  timeout and without drift.
"""

import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import make_atoms
from raspa3_b200.gcmc import beta_of, co2_component, fugacity_of, n2_component
from raspa3_b200.mixture import config5, random_mixture, total_energy
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu
BETA = beta_of(300.0)


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
        se = means[:, c].std(ddof=1) / math.sqrt(len(means))
        assert abs(means[:, c].mean() - t) < 4 * se + 0.03 * t, (c, means[:, c].mean(), t, se)


def framework_system(ctx, torch, kmax=6):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=kmax)
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
        host[idx] = buf.cpu().numpy()
    ew = native.Ewald(ctx, ff, scell)
    ew.set_framework(sfw)
    return ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host


def test_framework_mixture_drift_and_loading(ctx, torch, oracle):
    ff, ucell, ufw, scell, sfw, dims, sysg, ew, bufs, host = framework_system(ctx, torch)
    comps = [co2_component(), n2_component()]
    fug = [fugacity_of(1e6), fugacity_of(1e6)]
    runs = []
    for seed in range(4):
        mx = native.Mixture(sysg, ew, comps, BETA, fug, np.zeros((0, 3, 3)), np.zeros(0, dtype=np.int32),
                            max_molecules=256, seed=seed + 11)
        mx.set_state(0.0, ew.structure_factors(2))
        mx.run(3000, record=False)
        mx.run(20000, record=True)
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

    def one(seed):
        r, _, _, _ = oracle.mixture_run(ff, scell, comps, BETA, fug, np.zeros((0, 3, 3)), np.zeros(0, dtype=np.int32),
                                        23000, seed=seed, grids=host, grid_dims=dims, grid_cell=ucell,
                                        s_framework=s_fw, max_molecules=256)
        return r

    with ThreadPoolExecutor(4) as pool:
        ores = list(pool.map(one, range(4)))
    # the oracle records every move including the first 3000 (equilibration is short next to the run at this loading)
    cpu = np.array([[s / r["samples"] for s in r["sum_n"][:2]] for r in ores])
    for c in range(2):
        se = math.hypot(gpu[:, c].std(ddof=1) / 2, cpu[:, c].std(ddof=1) / 2)
        assert abs(gpu[:, c].mean() - cpu[:, c].mean()) < 4 * se + 0.05 * cpu[:, c].mean(), (c, gpu, cpu)


def test_large_mixture_runs_without_drift(ctx, torch):
    d = config5(ctx, torch)
    ff, comps = d["ff"], d["components"]
    e0 = total_energy(d["system"], d["ewald"], ff, comps, d["xyz"], d["comp"])
    sk0 = d["ewald"].structure_factors(0)
    mx = native.Mixture(d["system"], d["ewald"], comps, BETA, [fugacity_of(1e5), fugacity_of(1e5)], d["xyz"],
                        d["comp"], max_molecules=6000, seed=7)
    info = mx.info()
    assert info["n_kvectors"] == 3796
    mx.set_state(e0, sk0)
    mx.run(2000, record=True)
    r = mx.results()
    assert r["status"] == 0
    assert sum(r["accepted"]) > 0
    xyz, comp = mx.positions()
    e = total_energy(d["system"], d["ewald"], ff, comps, xyz, comp)
    assert abs(r["energy"] - e) < 1e-6 * max(1.0, abs(e)) + 1e-3, (r["energy"], e)
    mx.close()

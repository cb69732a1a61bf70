"""(a) Grid build on the GPU through the C-ABI vs the FP64 oracle (the reference's grid loop restated)."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import KELVIN_TO_ENERGY, make_atoms
from raspa3_b200.synthetic import (spacing_grid_dims, synthetic_forcefield, synthetic_framework)
from reference_systems import itq29, zeolite_forcefield

pytestmark = pytest.mark.gpu

E_LIMIT = 1e4 * KELVIN_TO_ENERGY  # the 1e-5 relative tolerance applies where |E| < 1e4 K
# Absolute floor of the energy channel's relative error, in K: 1e-5 relative to max(|E|, 1000 K), i.e. at most 0.01 K
# where the framework's terms (single terms up to ~5e5 K) cancel to |E| below 1000 K.
ENERGY_FLOOR_K = 1000.0


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def sample_points(dims, n, seed=7):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    pts = set(rng.integers(0, nx * ny * nz, size=n).tolist())
    # the duplicate periodic end-points and the corners
    for i in (0, nx - 1):
        for j in (0, ny - 1):
            for k in (0, nz - 1):
                pts.add(i + nx * (j + ny * k))
    return np.array(sorted(pts), dtype=np.int64)


def grid_errors(gpu, ref, beta_scale=1.0, energy_floor_k=ENERGY_FLOOR_K):
    """Errors of a grid against the FP64 oracle over the points with |E| < 1e4 K, per channel:
    * "rel":   energy channel: max |gpu - ref| / max(|E|, energy_floor_k) — relative to |E| itself, with an absolute
               floor for the points where the sum crosses zero; derivative channels (which cross zero everywhere):
               max |gpu - ref| / max(|ref|, RMS of the channel);
    * "boltz": sqrt(sum w (gpu - ref)^2 / sum w ref^2) with w = exp(-beta (E - E_min)) at 300 K, the Boltzmann-weighted
               relative error RASPA3 reports for its own grids (system_interpolation_grids.cpp:272-651).
    Returns (relative errors, boltzmann errors, number of points)."""
    mask = np.abs(ref[:, 0]) < E_LIMIT
    g, r = gpu[mask], ref[mask]
    d = np.abs(g - r)
    rms = np.sqrt(np.mean(r ** 2, axis=0)) + 1e-300
    scale = np.maximum(np.abs(r), rms)
    scale[:, 0] = np.maximum(np.abs(r[:, 0]), energy_floor_k * KELVIN_TO_ENERGY)
    rel = (d / scale).max(axis=0) if len(d) else np.zeros(8)
    beta = beta_scale / (300.0 * KELVIN_TO_ENERGY)
    w = np.exp(-beta * (r[:, 0] - r[:, 0].min()))[:, None] if len(d) else np.zeros((0, 1))
    boltz = np.sqrt(np.sum(w * d ** 2, axis=0) / (np.sum(w * r ** 2, axis=0) + 1e-300))
    return rel, boltz, int(mask.sum())


def test_methane_lj_fp64_full_grid_vs_oracle_sample(ctx, oracle):
    ff = synthetic_forcefield(charges=False)
    cell, atoms = synthetic_framework(ff)
    dims = spacing_grid_dims(cell)
    assert dims == (133, 133, 89)
    probe = ff.index("CH4")
    out, stats = ctx.grid_build(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64,
                                count_pairs=True)
    pts = sample_points(dims, 3000)
    ref = oracle.make_grid(0, ff, cell, atoms, probe, 12.0, dims, points=pts)
    gpu = out.reshape(-1, 8)[pts]
    # every sampled point, clamped overlaps included, to FP64 rounding
    rel = np.abs(gpu - ref) / np.maximum(np.abs(ref), 1.0)
    assert rel.max() < 1e-10, rel.max(axis=0)
    rel, boltz, n = grid_errors(gpu, ref)
    assert n > 20 and np.all(rel < 1e-10), rel
    assert stats["pair_count"] > 0 and stats["n_images"] > 0


def test_methane_pair_count_small_grid(ctx, oracle):
    ff = synthetic_forcefield(charges=False)
    cell, atoms = synthetic_framework(ff)
    dims = (21, 20, 14)
    probe = ff.index("CH4")
    _, stats = ctx.grid_build(0, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64, count_pairs=True)
    assert stats["pair_count"] == oracle.grid_pair_count(0, ff, cell, atoms, probe, 12.0, dims)


# FP32C acceptance: every channel within 1e-5 pointwise (energy relative to max(|E|, 1000 K), derivative channels
# relative to max(|value|, channel RMS)) and 1e-5 Boltzmann-weighted, for the Lennard-Jones grids and the unit-charge
# Ewald grid alike. The FP32C Ewald kernel evaluates the images near each brick in FP64 to get there (the FP64 mode is
# exact to 1e-10).
FP32C_TOL = {0: (1e-5, 1e-5), 1: (1e-5, 1e-5)}


@pytest.mark.parametrize("grid_type,probe_name", [(0, "C_co2"), (0, "O_co2"), (1, None)])
def test_charged_fp32c_vs_oracle_sample(ctx, oracle, grid_type, probe_name):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    dims = spacing_grid_dims(cell)
    probe = 0 if probe_name is None else ff.index(probe_name)
    out, _ = ctx.grid_build(grid_type, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP32C)
    pts = sample_points(dims, 3000, seed=11)
    ref = oracle.make_grid(grid_type, ff, cell, atoms, probe, 12.0, dims, points=pts)
    gpu = out.reshape(-1, 8)[pts]
    rel, boltz, n = grid_errors(gpu, ref, beta_scale=1.0 if grid_type == 0 else 0.35)
    print("fp32c", grid_type, probe_name, "pointwise", rel, "boltzmann", boltz)
    tol_pt, tol_bw = FP32C_TOL[grid_type]
    assert n > 100
    assert np.all(rel < tol_pt), rel
    assert np.all(boltz < tol_bw), boltz


@pytest.mark.parametrize("precision", [native.PRECISION_FP64, native.PRECISION_FP32C])
def test_itq29_small_full_grid(ctx, oracle, precision):
    """Known framework (zeolite force field: Si and O both Lennard-Jones), every point of a coarse grid."""
    ff = zeolite_forcefield(12.0, True, use_charge=True)
    cell, fw = itq29(ff)
    dims = (24, 24, 24)
    for grid_type, probe in ((0, ff.index("CH4")), (1, 0)):
        out, _ = ctx.grid_build(grid_type, ff, cell, fw, probe, 12.0, dims, precision)
        ref = oracle.make_grid(grid_type, ff, cell, fw, probe, 12.0, dims).reshape(-1, 8)
        rel, boltz, _ = grid_errors(out.reshape(-1, 8), ref)
        tol = 1e-10 if precision == native.PRECISION_FP64 else FP32C_TOL[grid_type][0]
        assert np.all(rel < tol), (grid_type, rel)
        # overlap-clamped points reproduce the reference clamp exactly
        clamp = ref[:, 0] == 2.0 * ff.overlap_criteria
        np.testing.assert_array_equal(out.reshape(-1, 8)[clamp, 0], ref[clamp, 0])


def test_triclinic_cell_fp64(ctx, oracle):
    """Triclinic branch: Cartesian tensors contracted with the cell vectors (framework_molecule_grid.cpp:244-279)."""
    ff = synthetic_forcefield(charges=True)
    rng = np.random.default_rng(3)
    cell = np.array([[14.0, 0.0, 0.0], [3.0, 13.0, 0.0], [2.0, 1.5, 12.5]])
    frac = rng.random((60, 3))
    pos = frac @ cell
    types = np.where(np.arange(60) % 3 == 0, ff.index("T"), ff.index("O")).astype(np.uint16)
    q = np.where(types == ff.index("T"), 2.05, -1.025)
    atoms = make_atoms(pos, types, q)
    dims = (12, 11, 10)
    for grid_type, probe in ((0, ff.index("CH4")), (1, 0)):
        out, _ = ctx.grid_build(grid_type, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64)
        ref = oracle.make_grid(grid_type, ff, cell, atoms, probe, 12.0, dims).reshape(-1, 8)
        rel, _, _ = grid_errors(out.reshape(-1, 8), ref)
        assert np.all(rel < 1e-9), (grid_type, rel)


def test_empty_framework_and_minimum_grid(ctx):
    ff = synthetic_forcefield(charges=False)
    cell = np.diag([10.0, 10.0, 10.0])
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    out, _ = ctx.grid_build(0, ff, cell, empty, ff.index("CH4"), 12.0, (2, 2, 2))
    assert out.shape == (64,) and np.all(out == 0.0)


def test_invalid_arguments_raise(ctx):
    ff = synthetic_forcefield(charges=False)
    cell, atoms = synthetic_framework(ff)
    with pytest.raises(native.RaspaGpuError):
        ctx.grid_build(0, ff, cell, atoms, 99, 12.0, (10, 10, 10))
    with pytest.raises(native.RaspaGpuError):
        ctx.grid_build(0, ff, cell, atoms, 2, 12.0, (1, 10, 10))


@pytest.mark.parametrize("precision", [native.PRECISION_FP64, native.PRECISION_FP32C])
def test_grid_build_set_matches_single_builds(ctx, precision):
    """rg_grid_build_set (Lennard-Jones probes fused two per kernel) gives the grids of separate rg_grid_build calls."""
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    dims = (45, 45, 30)
    types = [0, 0, 1]
    probes = [ff.index("C_co2"), ff.index("O_co2"), 0]
    outs = [torch.empty(8 * dims[0] * dims[1] * dims[2], dtype=torch.float64, device="cuda") for _ in types]
    hosts = [np.empty(8 * dims[0] * dims[1] * dims[2]) for _ in types]
    stats = ctx.grid_build_set(ff, cell, atoms, 12.0, dims, precision, types, probes, [o.data_ptr() for o in outs],
                               count_pairs=True, out_host=hosts)
    for g, (gt, pr) in enumerate(zip(types, probes)):
        ref, rs = ctx.grid_build(gt, ff, cell, atoms, pr, 12.0, dims, precision, count_pairs=True)
        np.testing.assert_array_equal(outs[g].cpu().numpy(), ref)
        np.testing.assert_array_equal(hosts[g], ref)
        assert stats[g]["pair_count"] == rs["pair_count"]


def _close(d, o, scale, rel=1e-9):
    return abs(d - o) <= rel * max(abs(o), scale, 1e-300)


def test_grid_validation_matches_oracle(ctx, oracle):
    """rg_grid_validate (the reference's grid test, system_interpolation_grids.cpp:240-651) on the device against the
    oracle at the same 2,000 points: every Boltzmann-weighted sum of the C_co2 VDW grid and of its charge term (0.70 e
    x the unit-charge Ewald grid), FP64 grids of the charged synthetic framework on a 0.5 A mesh in the 2x2x3 box.
    Tolerance 1e-9 of each sum's scale (for a sum of w x, sqrt(sum w x^2 sum w))."""
    torch = pytest.importorskip("torch")
    from raspa3_b200.synthetic import replicate

    ff = synthetic_forcefield(charges=True)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, _ = replicate(ucell, ufw, (2, 2, 3))
    dims = (41, 41, 28)
    probe = ff.index("C_co2")
    bufs = []
    for gt, pr in ((0, probe), (1, 0)):
        host, _ = ctx.grid_build(gt, ff, ucell, ufw, pr, 12.0, dims, native.PRECISION_FP64)
        bufs.append((host, torch.from_numpy(host).cuda()))
    pts = np.random.default_rng(7).random((2000, 3))
    beta = 1.0 / 300.0
    got = ctx.grid_validate(ff, ucell, ufw, scell, probe, dims, bufs[0][1].data_ptr(), bufs[1][1].data_ptr(), 0.70,
                            beta, points=pts)
    ref = oracle.grid_validate(ff, ucell, ufw, scell, probe, dims, bufs[0][0], bufs[1][0], 0.70, beta, pts)
    assert got["n_points"] == ref[34] == 2000
    assert got["n_points_charge"] == ref[35] > 100
    s = got["sums"]
    for base in (0, 17):
        o = ref[base:base + 17]
        assert _close(s[base], o[0], 0.0) and _close(s[base + 4], o[4], 0.0)
        for i in (1, 2):
            assert _close(s[base + i], o[i], np.sqrt(o[4] * o[0])), (base, i, s[base + i], o[i])
        assert _close(s[base + 3], o[3], o[4]), (base, s[base + 3], o[3])
        for a in range(3):
            g2 = o[14 + a]
            for i in (5 + a, 8 + a):
                assert _close(s[base + i], o[i], np.sqrt(g2 * o[0])), (base, i, s[base + i], o[i])
            assert _close(s[base + 11 + a], o[11 + a], g2), (base, a)
            assert _close(s[base + 14 + a], o[14 + a], 0.0), (base, a)
    # derived figures as the reference prints them
    assert abs(got["energy_relative_error"] - np.sqrt(ref[3] / ref[4])) <= 1e-9 * np.sqrt(ref[3] / ref[4])
    assert abs(got["charge_energy_table"] - ref[18] / ref[17]) <= 1e-9 * abs(ref[18] / ref[17])
    # Philox points: the same seed gives the same result, another seed another sample
    a = ctx.grid_validate(ff, ucell, ufw, scell, probe, dims, bufs[0][1].data_ptr(), bufs[1][1].data_ptr(), 0.70,
                          beta, n_points=50000, seed=3)
    b = ctx.grid_validate(ff, ucell, ufw, scell, probe, dims, bufs[0][1].data_ptr(), bufs[1][1].data_ptr(), 0.70,
                          beta, n_points=50000, seed=3)
    c = ctx.grid_validate(ff, ucell, ufw, scell, probe, dims, bufs[0][1].data_ptr(), bufs[1][1].data_ptr(), 0.70,
                          beta, n_points=50000, seed=4)
    assert a["sums"] == b["sums"] and a["n_points"] == 50000
    assert a["sums"] != c["sums"]
    assert abs(a["energy_relative_error"] - c["energy_relative_error"]) < 0.5 * a["energy_relative_error"]


def _triclinic_framework(ff, n=60, seed=3):
    rng = np.random.default_rng(seed)
    cell = np.array([[14.0, 0.0, 0.0], [3.0, 13.0, 0.0], [2.0, 1.5, 12.5]])
    pos = rng.random((n, 3)) @ cell
    types = np.where(np.arange(n) % 3 == 0, ff.index("T"), ff.index("O")).astype(np.uint16)
    q = np.where(types == ff.index("T"), 2.05, -1.025)
    return cell, make_atoms(pos, types, q)


@pytest.mark.parametrize("precision", [native.PRECISION_FP64, native.PRECISION_FP32C])
@pytest.mark.parametrize("cutoff,rc_vdw", [(9.0, 12.0), (12.0, 9.0), (7.0, 12.0)])
def test_cutoff_sizes_the_supercell(ctx, oracle, cutoff, rc_vdw, precision):
    """The `cutoff` argument sizes the reference's supercell (ceil(2 cutoff / width) cells, simulationbox.cpp:150-156)
    and the pair test uses cutOffFrameworkVDW (framework_molecule_grid.cpp:173, 202). With cutoff < cutOffFrameworkVDW
    (the reference builds the Ewald grid with cutOffCoulomb, system_interpolation_grids.cpp:211) the supercell's minimum
    image drops images within the pair cutoff; with cutoff > cutOffFrameworkVDW the supercell is only larger."""
    ff = synthetic_forcefield(rc=rc_vdw, charges=True)
    cell, atoms = synthetic_framework(ff)
    dims = (21, 20, 14)
    for grid_type, probe in ((1, 0), (0, ff.index("C_co2"))):
        out, st = ctx.grid_build(grid_type, ff, cell, atoms, probe, cutoff, dims, precision, count_pairs=True)
        ref = oracle.make_grid(grid_type, ff, cell, atoms, probe, cutoff, dims).reshape(-1, 8)
        assert st["pair_count"] == oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, cutoff, dims)
        rel, _, _ = grid_errors(out.reshape(-1, 8), ref)
        tol = 1e-10 if precision == native.PRECISION_FP64 else FP32C_TOL[grid_type][0]
        assert np.all(rel < tol), (grid_type, rel)
        if cutoff < rc_vdw:
            # the test has teeth: the supercell's minimum image drops pairs that a sum over every image within the
            # pair cutoff would keep
            assert st["pair_count"] < oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, rc_vdw, dims)


def test_cutoff_sizes_the_supercell_triclinic_fp64(ctx, oracle):
    """Triclinic cell with a supercell narrower than 2 rc along every axis: the minimum image in supercell fractions."""
    ff = synthetic_forcefield(rc=12.0, charges=True)
    cell, atoms = _triclinic_framework(ff)
    dims = (12, 11, 10)
    for grid_type, probe in ((1, 0), (0, ff.index("CH4"))):
        out, st = ctx.grid_build(grid_type, ff, cell, atoms, probe, 5.0, dims, native.PRECISION_FP64, count_pairs=True)
        ref = oracle.make_grid(grid_type, ff, cell, atoms, probe, 5.0, dims).reshape(-1, 8)
        assert st["pair_count"] == oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, 5.0, dims)
        rel, _, _ = grid_errors(out.reshape(-1, 8), ref)
        assert np.all(rel < 1e-9), (grid_type, rel)


def test_grid_build_set_reference_cutoffs_per_type(ctx, oracle):
    """rg_grid_build_set with cutoff <= 0 sizes each grid's supercell as the reference's grid loop does: cutOffCoulomb for
    the unit-charge Ewald grid, cutOffFrameworkVDW for the VDW grids (system_interpolation_grids.cpp:211, 236)."""
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(rc=12.0, charges=True)
    ff.cutoff_coulomb = 9.0
    cell, atoms = synthetic_framework(ff)
    dims = (21, 20, 14)
    types = [0, 0, 1]
    probes = [ff.index("C_co2"), ff.index("O_co2"), 0]
    n = 8 * dims[0] * dims[1] * dims[2]
    outs = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in types]
    ctx.grid_build_set(ff, cell, atoms, 0.0, dims, native.PRECISION_FP64, types, probes, [o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    for g, (gt, pr) in enumerate(zip(types, probes)):
        cut = 9.0 if gt == 1 else 12.0
        ref = oracle.make_grid(gt, ff, cell, atoms, pr, cut, dims).reshape(-1, 8)
        rel, _, _ = grid_errors(outs[g].cpu().numpy().reshape(-1, 8), ref)
        assert np.all(rel < 1e-10), (g, rel)


def test_nonpositive_cutoff_rejected(ctx):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    with pytest.raises(native.RaspaGpuError):
        ctx.grid_build(1, ff, cell, atoms, 0, 0.0, (4, 4, 4))

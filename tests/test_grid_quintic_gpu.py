"""Triquintic grids (27 values per point) on the GPU through the C-ABI vs the FP64 oracle, and device interpolation of
both schemes (rg_grid_build_triquintic, rg_grid_interpolate)."""

import math

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import KELVIN_TO_ENERGY, make_atoms
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu
E_LIMIT = 1e4 * KELVIN_TO_ENERGY


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


def channel_errors(gpu, ref):
    """Per channel: max |gpu - ref| / max(|ref|, RMS of the channel) over the points with |E| < 1e4 K."""
    g, r = gpu.reshape(-1, 27), ref.reshape(-1, 27)
    mask = np.abs(r[:, 0]) < E_LIMIT
    g, r = g[mask], r[mask]
    rms = np.sqrt(np.mean(r ** 2, axis=0)) + 1e-300
    return (np.abs(g - r) / np.maximum(np.abs(r), rms)).max(axis=0), int(mask.sum())


def triclinic_system(ff, n=60, seed=3):
    rng = np.random.default_rng(seed)
    cell = np.array([[14.0, 0.0, 0.0], [3.0, 13.0, 0.0], [2.0, 1.5, 12.5]])
    pos = rng.random((n, 3)) @ cell
    types = np.where(np.arange(n) % 3 == 0, ff.index("T"), ff.index("O")).astype(np.uint16)
    q = np.where(types == ff.index("T"), 2.05, -1.025)
    return cell, make_atoms(pos, types, q)


@pytest.mark.parametrize("grid_type", [native.GRID_LENNARD_JONES, native.GRID_EWALD_REAL])
@pytest.mark.parametrize("reference_rectangular", [False, True])
def test_rectangular_triquintic_vs_oracle(ctx, oracle, grid_type, reference_rectangular):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    dims = (12, 11, 9)
    probe = ff.index("CH4") if grid_type == native.GRID_LENNARD_JONES else 0
    out, stats = ctx.grid_build_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims,
                                           reference_rectangular=reference_rectangular, count_pairs=True)
    ref = oracle.make_grid_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims,
                                      reference_rectangular=reference_rectangular)
    err, n = channel_errors(out, ref)
    assert n >= 30
    assert np.all(err < 1e-9), err
    # overlap clamp (interpolation_energy_grid.cpp:3937-3955): energy 2 x criterion, first derivatives clamped, the
    # rest zero
    clamp = ref.reshape(-1, 27)[:, 0] == 2.0 * ff.overlap_criteria
    o, r = out.reshape(-1, 27)[clamp], ref.reshape(-1, 27)[clamp]
    np.testing.assert_array_equal(o[:, 0], r[:, 0])
    np.testing.assert_allclose(o[:, 1:4], r[:, 1:4], rtol=1e-12)
    assert np.all(o[:, 4:] == 0.0)
    assert stats["pair_count"] == oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, 12.0, dims)


@pytest.mark.parametrize("grid_type", [native.GRID_LENNARD_JONES, native.GRID_EWALD_REAL])
def test_triclinic_triquintic_vs_oracle(ctx, oracle, grid_type):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = triclinic_system(ff)
    dims = (10, 9, 9)
    probe = ff.index("CH4") if grid_type == native.GRID_LENNARD_JONES else 0
    out, _ = ctx.grid_build_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims)
    ref = oracle.make_grid_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims)
    err, n = channel_errors(out, ref)
    assert n >= 30
    assert np.all(err < 1e-9), err
    # the reference flag changes nothing for a triclinic cell
    out2, _ = ctx.grid_build_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims, reference_rectangular=True)
    np.testing.assert_array_equal(out2, out)


def test_interpolation_of_both_schemes_vs_oracle(ctx, oracle, torch):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = triclinic_system(ff, n=45, seed=8)
    dims = (15, 14, 13)
    probe = ff.index("CH4")
    rng = np.random.default_rng(4)
    pos = rng.random((300, 3)) @ cell + rng.normal(size=(300, 3))  # some outside the cell: wrapped by fract
    # triquintic
    q = torch.empty(27 * math.prod(dims), dtype=torch.float64, device="cuda")
    ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims, out_device=q.data_ptr(),
                              host=False)
    ctx.synchronize()
    qh = q.cpu().numpy()
    e, g = ctx.grid_interpolate(native.SCHEME_TRIQUINTIC, q.data_ptr(), dims, cell, pos)
    inv = np.linalg.inv(cell)
    grid = qh.reshape(dims[2], dims[1], dims[0], 27)
    for t in range(len(pos)):
        v, gr = oracle.interpolate_triquintic(qh, dims, cell, pos[t])
        # the oracle sums the reference's monomial form, whose rounding grows with the largest corner value (cells
        # next to overlap-clamped points hold 2e6): tolerance from the value and from the cell's corner data
        s = (pos[t] @ inv) % 1.0
        i0 = [min(int(s[d] * (dims[d] - 1)), dims[d] - 2) for d in range(3)]
        xmax = np.abs(grid[i0[2]:i0[2] + 2, i0[1]:i0[1] + 2, i0[0]:i0[0] + 2]).max()
        assert abs(e[t] - v) < 1e-9 * max(1.0, abs(v)) + 1e-11 * xmax, (t, e[t], v, xmax)
        np.testing.assert_allclose(g[t], gr, rtol=0, atol=1e-8 * max(1.0, np.abs(gr).max()) + 1e-10 * xmax)
    # tricubic through the same entry point
    c = torch.empty(8 * math.prod(dims), dtype=torch.float64, device="cuda")
    ctx.grid_build(native.GRID_LENNARD_JONES, ff, cell, atoms, probe, 12.0, dims, native.PRECISION_FP64,
                   out_device=c.data_ptr(), host=False)
    ctx.synchronize()
    ch = c.cpu().numpy()
    e8, g8 = ctx.grid_interpolate(native.SCHEME_TRICUBIC, c.data_ptr(), dims, cell, pos)
    for t in range(len(pos)):
        v = oracle.interpolate(ch, dims, cell, pos[t])
        assert abs(e8[t] - v) < 1e-9 * max(1.0, abs(v))
    assert np.all(np.isfinite(g8))


def test_triquintic_interpolates_more_accurately_than_tricubic(ctx, oracle, torch):
    """On the same grid points the triquintic interpolant (second derivatives stored) is closer to the analytical
    energy than the tricubic one: Boltzmann-weighted relative error at 300 K over random points."""
    ff = synthetic_forcefield(charges=False)
    ucell, uatoms = synthetic_framework(ff)
    dims = (41, 41, 28)
    probe = ff.index("CH4")
    q = torch.empty(27 * math.prod(dims), dtype=torch.float64, device="cuda")
    c = torch.empty(8 * math.prod(dims), dtype=torch.float64, device="cuda")
    ctx.grid_build_triquintic(0, ff, ucell, uatoms, probe, 12.0, dims, out_device=q.data_ptr(), host=False)
    ctx.grid_build(0, ff, ucell, uatoms, probe, 12.0, dims, native.PRECISION_FP64, out_device=c.data_ptr(),
                   host=False)
    ctx.synchronize()
    # most of this dense framework is inaccessible to methane: keep the random points whose tricubic estimate is
    # below 2e3 K, then compare where the analytical energy is below 1e3 K
    rng = np.random.default_rng(9)
    pos = rng.random((200000, 3)) @ ucell
    est, _ = ctx.grid_interpolate(native.SCHEME_TRICUBIC, c.data_ptr(), dims, ucell, pos, gradients=False)
    pos = pos[est < 2e3 * KELVIN_TO_ENERGY][:2000]
    eq, _ = ctx.grid_interpolate(native.SCHEME_TRIQUINTIC, q.data_ptr(), dims, ucell, pos, gradients=False)
    ec, _ = ctx.grid_interpolate(native.SCHEME_TRICUBIC, c.data_ptr(), dims, ucell, pos, gradients=False)
    reps = [math.ceil(24.0 / w) for w in np.diag(ucell)]
    scell, satoms = replicate(ucell, uatoms, reps)
    full = np.array([oracle.tricubic_fractional(0, ff, scell, p, probe, ucell, satoms)[0] for p in pos])
    ok = full < 1e3 * KELVIN_TO_ENERGY
    w = np.exp(-full[ok] / (300.0 * KELVIN_TO_ENERGY) + full[ok].min() / (300.0 * KELVIN_TO_ENERGY))
    err_q = math.sqrt(np.sum(w * (eq[ok] - full[ok]) ** 2) / np.sum(w * full[ok] ** 2))
    err_c = math.sqrt(np.sum(w * (ec[ok] - full[ok]) ** 2) / np.sum(w * full[ok] ** 2))
    assert ok.sum() > 100
    assert err_q < err_c, (err_q, err_c)


def test_triquintic_argument_errors(ctx, torch):
    ff = synthetic_forcefield(charges=False)
    cell, atoms = synthetic_framework(ff)
    with pytest.raises(native.RaspaGpuError, match="Lennard-Jones or Ewald-real"):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES_REPULSION, ff, cell, atoms, ff.index("CH4"), 12.0,
                                  (4, 4, 4))
    with pytest.raises(native.RaspaGpuError):
        ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell, atoms, ff.index("CH4"), 12.0, (1, 4, 4))
    buf = torch.zeros(27 * 64, dtype=torch.float64, device="cuda")
    with pytest.raises(native.RaspaGpuError, match="scheme"):
        ctx.grid_interpolate(9, buf.data_ptr(), (4, 4, 4), cell, np.zeros((1, 3)))


def test_trial_energies_with_triquintic_grids(ctx, oracle):
    """rg_cbmc_external_energies on a system whose grids are triquintic: the grid branch of each trial atom is the
    triquintic interpolant of its VDW grid plus q times that of the unit-charge Ewald grid."""
    ff = synthetic_forcefield(charges=True)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, sfw = replicate(ucell, ufw, (2, 2, 3))
    dims = (34, 34, 23)
    sysg = native.System(ctx, ff, scell, sfw)
    sysg.set_interpolation_scheme(native.SCHEME_TRIQUINTIC)
    host = {}
    for name, gt in (("C_co2", native.GRID_LENNARD_JONES), ("O_co2", native.GRID_LENNARD_JONES),
                     (None, native.GRID_EWALD_REAL)):
        idx = ff.index(name) if name else ff.n_types
        g, _ = ctx.grid_build_triquintic(gt, ff, ucell, ufw, idx if name else 0, 12.0, dims)
        sysg.set_grid(idx, ucell, dims, g)
        host[idx] = g
    with pytest.raises(native.RaspaGpuError, match="before the first grid"):
        sysg.set_interpolation_scheme(native.SCHEME_TRICUBIC)
    rng = np.random.default_rng(12)
    for name in ("C_co2", "O_co2"):
        t = ff.index(name)
        q = float(ff.pseudo_atoms[t].charge)
        pos = rng.random((40, 3)) @ scell
        trials = make_atoms(pos, t, q, molecule_ids=np.zeros(40, dtype=np.int64))
        res = sysg.external_energies(trials, 1)
        for i, r in enumerate(res):
            e_vdw, _ = oracle.interpolate_triquintic(host[t], dims, ucell, pos[i])
            e_q, _ = oracle.interpolate_triquintic(host[ff.n_types], dims, ucell, pos[i])
            assert bool(r.overlap) == (e_vdw > ff.overlap_criteria)
            if r.overlap:
                continue
            assert r.framework_vdw == pytest.approx(e_vdw, rel=1e-10, abs=1e-8)
            assert r.framework_charge == pytest.approx(q * e_q, rel=1e-10, abs=1e-8)
    sysg.close()


def _close(a, b, scale):
    return abs(a - b) <= 1e-9 * max(abs(b), scale, 1e-300)


def test_triquintic_grid_test_matches_oracle(ctx, oracle, torch):
    """rg_grid_validate_triquintic (the reference's grid test with the triquintic scheme, Hessians included) against
    the oracle at the same 600 points: every Boltzmann-weighted sum of the C_co2 VDW grid and of its charge term
    (0.70 e x the unit-charge Ewald grid), charged synthetic framework on a 0.5 A mesh, 2x2x3 box. Tolerance 1e-9 of each
    sum's scale (for a sum of w x, sqrt(sum w x^2 sum w))."""
    ff = synthetic_forcefield(charges=True)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, _ = replicate(ucell, ufw, (2, 2, 3))
    dims = (41, 41, 28)
    probe = ff.index("C_co2")
    bufs = []
    for gt, pr in ((native.GRID_LENNARD_JONES, probe), (native.GRID_EWALD_REAL, 0)):
        host, _ = ctx.grid_build_triquintic(gt, ff, ucell, ufw, pr, 12.0, dims)
        bufs.append((host, torch.from_numpy(host).cuda()))
    pts = np.random.default_rng(7).random((600, 3))
    beta = 1.0 / 300.0
    got = ctx.grid_validate_triquintic(ff, ucell, ufw, scell, probe, dims, bufs[0][1].data_ptr(),
                                       bufs[1][1].data_ptr(), 0.70, beta, points=pts)
    ref = oracle.grid_validate_triquintic(ff, ucell, ufw, scell, probe, dims, bufs[0][0], bufs[1][0], 0.70, beta, pts)
    assert got["n_points"] == ref[34] == 600
    assert got["n_points_charge"] == ref[35] > 30
    s, hs = got["sums"], got["hessian"]["sums"]
    for base, hbase in ((0, 0), (17, 24)):
        o, oh = ref[base:base + 17], ref[36 + hbase:36 + hbase + 24]
        w = o[0]
        assert _close(s[base], w, 0.0) and _close(s[base + 4], o[4], 0.0)
        for i in (1, 2):
            assert _close(s[base + i], o[i], np.sqrt(o[4] * w)), (base, i, s[base + i], o[i])
        assert _close(s[base + 3], o[3], o[4])
        for a in range(3):
            g2 = o[14 + a]
            for i in (5 + a, 8 + a):
                assert _close(s[base + i], o[i], np.sqrt(g2 * w)), (base, i, s[base + i], o[i])
            assert _close(s[base + 11 + a], o[11 + a], g2)
            assert _close(s[base + 14 + a], o[14 + a], 0.0)
        for q in range(6):
            h2 = oh[18 + q]
            for i in (q, 6 + q):
                assert _close(hs[hbase + i], oh[i], np.sqrt(h2 * w)), (base, q, i, hs[hbase + i], oh[i])
            assert _close(hs[hbase + 12 + q], oh[12 + q], h2), (base, q)
            assert _close(hs[hbase + 18 + q], oh[18 + q], 0.0), (base, q)
    h = got["hessian"]
    assert abs(h["hessian_relative_error"][0] - np.sqrt(ref[36 + 12] / ref[36 + 18])) <= \
        1e-9 * np.sqrt(ref[36 + 12] / ref[36 + 18])
    # the triquintic grid's VDW energy error is well below the tricubic grid's on the same mesh
    c = torch.from_numpy(ctx.grid_build(0, ff, ucell, ufw, probe, 12.0, dims, native.PRECISION_FP64)[0]).cuda()
    tri = ctx.grid_validate(ff, ucell, ufw, scell, probe, dims, c.data_ptr(), None, 0.0, beta, points=pts)
    assert got["energy_relative_error"] < tri["energy_relative_error"]


def test_triquintic_edge_cases(ctx, oracle, torch):
    """An empty framework gives an all-zero grid, the smallest grid (2 x 2 x 2 points) matches the oracle, and the
    triquintic grid test of no points returns zero counts."""
    ff = synthetic_forcefield(charges=True)
    cell = np.diag([10.0, 11.0, 12.0])
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    for gt in (native.GRID_LENNARD_JONES, native.GRID_EWALD_REAL):
        out, _ = ctx.grid_build_triquintic(gt, ff, cell, empty, ff.index("CH4"), 12.0, (3, 3, 2))
        assert out.shape == (27 * 18,) and np.all(out == 0.0)
    cell2, atoms = triclinic_system(ff, n=12, seed=5)
    out, _ = ctx.grid_build_triquintic(native.GRID_LENNARD_JONES, ff, cell2, atoms, ff.index("CH4"), 12.0, (2, 2, 2))
    ref = oracle.make_grid_triquintic(0, ff, cell2, atoms, ff.index("CH4"), 12.0, (2, 2, 2))
    err, _ = channel_errors(out, ref)
    assert np.all(err < 1e-9)
    buf = torch.from_numpy(out).cuda()
    r = ctx.grid_validate_triquintic(ff, cell2, atoms, cell2, ff.index("CH4"), (2, 2, 2), buf.data_ptr(),
                                     points=np.zeros((0, 3)))
    assert r["n_points"] == 0 and r["n_points_charge"] == 0


# FP32C acceptance (stated; measured on B200 4.8e-6 and 1.6e-5): every channel within 2e-5 of max(|value|, channel
# RMS) for the Lennard-Jones grid and within 5e-5 for the unit-charge Ewald grid, whose large +2.05 / -1.025 e terms
# cancel.
TQ_FP32C_TOL = {native.GRID_LENNARD_JONES: 2e-5, native.GRID_EWALD_REAL: 5e-5}


@pytest.mark.parametrize("grid_type", [native.GRID_LENNARD_JONES, native.GRID_EWALD_REAL])
@pytest.mark.parametrize("triclinic", [False, True])
def test_triquintic_fp32c_vs_oracle(ctx, oracle, grid_type, triclinic):
    ff = synthetic_forcefield(charges=True)
    if triclinic:
        cell, atoms = triclinic_system(ff)
        dims = (10, 9, 9)
    else:
        cell, atoms = synthetic_framework(ff)
        dims = (12, 11, 9)
    probe = ff.index("CH4") if grid_type == native.GRID_LENNARD_JONES else 0
    out, _ = ctx.grid_build_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims, fp32c=True)
    ref = oracle.make_grid_triquintic(grid_type, ff, cell, atoms, probe, 12.0, dims)
    err, n = channel_errors(out, ref)
    print("triquintic fp32c", grid_type, triclinic, "max channel error", err.max(), "points", n)
    assert n >= 30
    assert np.all(err < TQ_FP32C_TOL[grid_type]), err


@pytest.mark.parametrize("triclinic", [False, True])
def test_triquintic_cutoff_sizes_the_supercell(ctx, oracle, triclinic):
    """As for the tricubic build: the cutoff argument sizes the reference's supercell, whose minimum image drops pairs
    within the pair cutoff when it is narrower than twice that cutoff."""
    ff = synthetic_forcefield(charges=True)
    cell, atoms = triclinic_system(ff) if triclinic else synthetic_framework(ff)
    cutoff = 5.0 if triclinic else 9.0
    dims = (9, 8, 8)
    for grid_type, probe in ((native.GRID_EWALD_REAL, 0), (native.GRID_LENNARD_JONES, ff.index("CH4"))):
        out, stats = ctx.grid_build_triquintic(grid_type, ff, cell, atoms, probe, cutoff, dims, count_pairs=True)
        ref = oracle.make_grid_triquintic(grid_type, ff, cell, atoms, probe, cutoff, dims)
        err, n = channel_errors(out, ref)
        assert n >= 10 and np.all(err < 1e-9), (n, err)
        assert stats["pair_count"] == oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, cutoff, dims)
        assert stats["pair_count"] < oracle.grid_pair_count(grid_type, ff, cell, atoms, probe, 12.0, dims)

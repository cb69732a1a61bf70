"""The grid build that allocates nothing (rg_grid_build_noalloc), for callers that cannot allocate device memory,
checked through the C-ABI against the regular entry point rg_grid_build on the same inputs, on two calls in a row.

Collected last on purpose: if it fails, a run that stops at the first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ATOM_DTYPE, box_struct, ff_struct, make_atoms
from raspa3_b200.synthetic import synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu


def noalloc_build(torch, ff, cell, atoms, grid_type, probe, dims, precision, stream=None, cutoff=12.0):
    nx, ny, nz = dims
    out = torch.full((8 * nx * ny * nz,), float("nan"), dtype=torch.float64, device="cuda")
    atoms = np.ascontiguousarray(atoms, dtype=ATOM_DTYPE)
    ffs, box = ff_struct(ff), box_struct(cell)
    stats = native.GridStats()
    st = native.lib().rg_grid_build_noalloc(0, stream, grid_type, ctypes.byref(ffs), ctypes.byref(box),
                                            ctypes.c_void_p(atoms.ctypes.data), len(atoms), probe, cutoff, nx, ny, nz,
                                            precision, ctypes.c_void_p(out.data_ptr()), ctypes.byref(stats))
    torch.cuda.synchronize()
    return st, out.cpu().numpy(), stats


def test_noalloc_grid_build_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff, seed=42)
    dims = (40, 40, 27)
    ctx = native.Context(0)
    try:
        # two calls in a row with different work: the shared scratch keeps the first call's images and count
        for grid_type, probe, precision, tol in ((1, 0, native.PRECISION_FP64, 1e-10),
                                                 (0, ff.index("C_co2"), native.PRECISION_FP32C, 1e-5)):
            st, got, stats = noalloc_build(torch, ff, cell, atoms, grid_type, probe, dims, precision)
            assert st == native.RG_OK
            ref, ref_stats = ctx.grid_build(grid_type, ff, cell, atoms, probe, 12.0, dims, precision,
                                            count_pairs=True)
            assert np.all(np.isfinite(got))
            rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1.0)
            assert rel.max() < tol, rel.max()
            assert stats.pair_count == ref_stats["pair_count"]
            assert stats.n_images == ref_stats["n_images"]
    finally:
        ctx.close()


def test_noalloc_rejects_more_images_than_its_array_holds():
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(charges=True)
    # 6000 charged atoms in a 10 A cell: ~27 images each, far beyond the 32768 the scratch array holds
    rng = np.random.default_rng(0)
    cell = np.diag([10.0, 10.0, 10.0])
    atoms = make_atoms(rng.random((6000, 3)) * 10.0, ff.index("O"), -1.025)
    st, _, _ = noalloc_build(torch, ff, cell, atoms, 1, 0, (4, 4, 4), native.PRECISION_FP64)
    assert st == 1  # RG_ERR_INVALID_ARGUMENT


def test_noalloc_on_a_caller_stream_with_a_clipped_supercell():
    """On a caller's non-default stream the image copies, the counter reset and the kernel are ordered on that stream;
    a cutoff below the pair cutoff sizes the supercell as in rg_grid_build. The caller's current device is kept."""
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff, seed=42)
    dims = (30, 30, 20)
    ctx = native.Context(0)
    try:
        stream = torch.cuda.Stream()
        for grid_type, probe in ((1, 0), (0, ff.index("O_co2"))):
            st, got, stats = noalloc_build(torch, ff, cell, atoms, grid_type, probe, dims, native.PRECISION_FP64,
                                           stream=ctypes.c_void_p(stream.cuda_stream), cutoff=9.0)
            assert st == native.RG_OK
            assert torch.cuda.current_device() == 0
            ref, ref_stats = ctx.grid_build(grid_type, ff, cell, atoms, probe, 9.0, dims, native.PRECISION_FP64,
                                            count_pairs=True)
            rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1.0)
            assert rel.max() < 1e-10, rel.max()
            assert stats.pair_count == ref_stats["pair_count"]
    finally:
        ctx.close()


def test_noalloc_at_exactly_its_image_limit():
    """32768 images fill the array exactly (the flush after the last full staging chunk still runs); one more atom is
    rejected. Atoms inside the middle fifth of a 30 A cubic cell have exactly one periodic image within 12 A of the
    unit cell each."""
    torch = pytest.importorskip("torch")
    ff = synthetic_forcefield(charges=True)
    rng = np.random.default_rng(1)
    cell = np.diag([30.0, 30.0, 30.0])
    n = 32768
    pos = (0.4 + 0.2 * rng.random((n + 1, 3))) * 30.0
    q = np.where(np.arange(n + 1) % 2 == 0, 1.0, -1.0)
    atoms = make_atoms(pos, ff.index("O"), q)
    dims = (4, 4, 4)
    st, got, stats = noalloc_build(torch, ff, cell, atoms[:n], 1, 0, dims, native.PRECISION_FP64)
    assert st == native.RG_OK and stats.n_images == n
    ctx = native.Context(0)
    try:
        ref, ref_stats = ctx.grid_build(1, ff, cell, atoms[:n], 0, 12.0, dims, native.PRECISION_FP64, count_pairs=True)
    finally:
        ctx.close()
    assert ref_stats["n_images"] == n and stats.pair_count == ref_stats["pair_count"]
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    st, _, _ = noalloc_build(torch, ff, cell, atoms, 1, 0, dims, native.PRECISION_FP64)
    assert st == 1  # RG_ERR_INVALID_ARGUMENT

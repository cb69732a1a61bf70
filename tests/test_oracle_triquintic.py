"""The oracle of the triquintic scheme (27 values per grid point): its interpolating polynomial against the
reference's own coefficient map, and its grid values against independent checks.

* interpolants.json holds the reference's computeCoefficients maps (interpolation_energy_grid.cpp:193-358 and
  :2116-3500) applied to seeded random corner data; the oracle's regenerated maps must reproduce them.
* The rectangular branch of calculateTriquinticFractionalAtPosition (framework_molecule_grid.cpp:568-683) restated
  exactly equals the triclinic branch (:684-812) for the same cell; the reference's two deviations of the rectangular
  branch change channels 2, 3 and 26 only.
* Every channel is the lattice derivative of a lower channel: central finite differences along the lattice vectors.
"""

import json
import math
import os

import numpy as np
import pytest

from raspa3_b200.forcefield import make_atoms
from raspa3_b200.synthetic import replicate, synthetic_forcefield

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "interpolants.json")
ORDERS = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2),
          (2, 1, 0), (2, 0, 1), (1, 2, 0), (1, 1, 1), (0, 2, 1), (1, 0, 2), (0, 1, 2), (2, 2, 0), (2, 0, 2), (0, 2, 2),
          (2, 1, 1), (1, 2, 1), (1, 1, 2), (2, 2, 1), (2, 1, 2), (1, 2, 2), (2, 2, 2)]


def widths(cell):
    cell = np.asarray(cell)
    v = abs(np.linalg.det(cell))
    return [v / np.linalg.norm(np.cross(cell[(a + 1) % 3], cell[(a + 2) % 3])) for a in range(3)]


def small_system(triclinic, seed=5, n=6):
    ff = synthetic_forcefield(charges=True)
    if triclinic:
        cell = np.array([[14.0, 0.0, 0.0], [3.0, 13.0, 0.0], [2.0, 1.5, 12.5]])
    else:
        cell = np.diag([14.0, 13.0, 12.5])
    rng = np.random.default_rng(seed)
    pos = rng.random((n, 3)) @ cell
    types = np.where(np.arange(n) % 3 == 0, ff.index("T"), ff.index("O")).astype(np.uint16)
    q = np.where(types == ff.index("T"), 2.05, -1.025)
    atoms = make_atoms(pos, types, q)
    reps = [math.ceil(2.0 * 12.0 / w) for w in widths(cell)]
    scell, satoms = replicate(cell, atoms, reps)
    return ff, cell, atoms, scell, satoms


def clear_point(cell, atoms, rng, rmin=4.0):
    """A point at least rmin from every periodic image of the atoms."""
    inv = np.linalg.inv(cell)
    xyz = np.stack([atoms["x"], atoms["y"], atoms["z"]], axis=1)
    for _ in range(10000):
        p = rng.random(3) @ cell
        d = (p - xyz) @ inv
        d -= np.round(d)
        if np.min(np.linalg.norm(d @ cell, axis=1)) > rmin:
            return p
    raise AssertionError("no clear point")


@pytest.mark.parametrize("scheme", [8, 27])
def test_interpolants_match_reference_coefficient_maps(oracle, scheme):
    cases = json.load(open(GOLDEN))["cases"][str(scheme)]
    assert len(cases) >= 8
    for c in cases:
        v, ds = oracle.interpolant_from_corners(scheme, c["X"], c["s"])
        scale = max(1.0, abs(c["value"]), float(np.abs(c["ds"]).max()))
        assert abs(v - c["value"]) < 1e-11 * scale
        np.testing.assert_allclose(ds, c["ds"], rtol=0, atol=1e-11 * scale)


def test_triquintic_polynomial_reproduces_corner_data(oracle):
    rng = np.random.default_rng(3)
    X = rng.normal(size=216)
    for corner in range(8):
        s = [corner & 1, (corner >> 1) & 1, (corner >> 2) & 1]
        v, ds = oracle.interpolant_from_corners(27, X, s)
        # sums of 216 monomials with coefficients in the thousands: agreement to rounding
        assert abs(v - X[corner]) < 1e-10
        np.testing.assert_allclose(ds, [X[8 + corner], X[16 + corner], X[24 + corner]], atol=1e-9)
    m = oracle.triquintic_matrix()
    assert np.all(m * 8 == np.rint(m * 8))


@pytest.mark.parametrize("grid_type", [0, 1])
def test_rectangular_branch_equals_triclinic_branch(oracle, grid_type):
    ff, cell, atoms, scell, satoms = small_system(triclinic=False)
    probe = ff.index("CH4") if grid_type == 0 else 0
    rng = np.random.default_rng(11)
    for _ in range(3):
        p = clear_point(cell, atoms, rng, rmin=2.5)
        rect = oracle.triquintic_fractional(grid_type, ff, scell, p, probe, cell, satoms, triclinic=False)
        tri = oracle.triquintic_fractional(grid_type, ff, scell, p, probe, cell, satoms, triclinic=True)
        scale = np.abs(tri) + 1e-9 * np.abs(tri).max()
        assert np.all(np.abs(rect - tri) <= 1e-10 * scale), np.abs(rect - tri) / scale
        compat = oracle.triquintic_fractional(grid_type, ff, scell, p, probe, cell, satoms, reference_rectangular=True,
                                              triclinic=False)
        same = [l for l in range(27) if l not in (2, 3, 26)]
        np.testing.assert_array_equal(compat[same], rect[same])
        assert compat[2] == pytest.approx(rect[2] * cell[0, 0] / cell[1, 1], rel=1e-13)
        assert compat[3] == pytest.approx(rect[3] * cell[0, 0] / cell[2, 2], rel=1e-13)
        assert compat[26] != rect[26]


@pytest.mark.parametrize("grid_type", [0, 1])
def test_channels_are_lattice_derivatives(oracle, grid_type):
    """channel(o) = d/ds_a channel(o - e_a) for an axis a with o_a > 0 (central differences, h = 1e-5 in fractions)."""
    ff, cell, atoms, scell, satoms = small_system(triclinic=True)
    probe = ff.index("CH4") if grid_type == 0 else 0
    rng = np.random.default_rng(2)
    p = clear_point(cell, atoms, rng, rmin=4.0)
    h = 1e-5

    def chans(x):
        return oracle.triquintic_fractional(grid_type, ff, scell, x, probe, cell, satoms)

    base = chans(p)
    up = [chans(p + h * cell[a]) for a in range(3)]
    dn = [chans(p - h * cell[a]) for a in range(3)]
    for l, o in enumerate(ORDERS):
        if l == 0:
            continue
        a = max(range(3), key=lambda ax: o[ax])
        lower = ORDERS.index(tuple(o[ax] - (ax == a) for ax in range(3)))
        fd = (up[a][lower] - dn[a][lower]) / (2 * h)
        scale = max(abs(base[l]), 1e-6 * np.abs(base).max())
        assert abs(fd - base[l]) < 2e-5 * scale, (l, o, fd, base[l])


def test_grid_build_and_interpolation_at_grid_points(oracle):
    ff, cell, atoms, _, _ = small_system(triclinic=True, n=9)
    dims = (7, 6, 6)
    grid = oracle.make_grid_triquintic(0, ff, cell, atoms, ff.index("CH4"), 12.0, dims).reshape(-1, 27)
    nx, ny, nz = dims
    inv = np.linalg.inv(cell)
    for flat in (0, 1 + nx * (2 + ny * 3), 5 + nx * (4 + ny * 2)):
        i, j, k = flat % nx, (flat // nx) % ny, flat // (nx * ny)
        s = np.array([i / (nx - 1), j / (ny - 1), k / (nz - 1)])
        v, grad = oracle.interpolate_triquintic(grid.reshape(-1), dims, cell, s @ cell + 1e-12)
        g = grid[flat]
        assert v == pytest.approx(g[0], rel=1e-9, abs=1e-9)
        # Cartesian gradient = inverse-cell transpose times d/ds, and d/ds = channel * (n - 1)
        ds = np.array([g[1] * (nx - 1), g[2] * (ny - 1), g[3] * (nz - 1)])
        np.testing.assert_allclose(grad, inv @ ds, rtol=1e-7, atol=1e-7 * np.abs(ds).max())
    # the point list gives the same values as the full grid
    pts = np.array([0, 17, 100, nx * ny * nz - 1])
    some = oracle.make_grid_triquintic(0, ff, cell, atoms, ff.index("CH4"), 12.0, dims, points=pts)
    np.testing.assert_array_equal(some, grid[pts])

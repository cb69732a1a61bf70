"""The oracle of the grid test (System::createFrameworkInterpolationGrids, system_interpolation_grids.cpp:240-651):
both gradients it compares, the interpolant's (interpolateHessian) and the analytical one
(calculateTricubicFractionalAtPosition mapped to Cartesian), agree with central finite differences of their energies.
"""

import numpy as np
import pytest

from raspa3_b200.forcefield import ENERGY_TO_KELVIN
from raspa3_b200.synthetic import replicate, synthetic_forcefield, synthetic_framework


def test_oracle_gradients_match_finite_differences(oracle):
    ff = synthetic_forcefield(charges=True)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, _ = replicate(ucell, ufw, (2, 2, 3))
    dims = (21, 21, 14)
    probe = ff.index("CH4")
    grid = oracle.make_grid(0, ff, ucell, ufw, probe, 12.0, dims)
    inv = np.linalg.inv(scell)
    rng = np.random.default_rng(11)
    h = 1e-5
    checked = 0
    for _ in range(400):
        if checked == 4:
            break
        pos = rng.random(3) @ scell
        one = oracle.grid_validate(ff, ucell, ufw, scell, probe, dims, grid, None, 0.0, 0.0, [pos @ inv])
        if one[2] > 1e4:  # inside the framework (most of this dense cell for methane): skip steep overlap regions
            continue
        checked += 1
        fd_table, fd_full = [], []
        for a in range(3):
            d = np.zeros(3)
            d[a] = h
            e_up = oracle.interpolate(grid, dims, ucell, pos + d)
            e_dn = oracle.interpolate(grid, dims, ucell, pos - d)
            fd_table.append((e_up - e_dn) / (2 * h) * ENERGY_TO_KELVIN)
            up = oracle.grid_validate(ff, ucell, ufw, scell, probe, dims, grid, None, 0.0, 0.0, [(pos + d) @ inv])
            dn = oracle.grid_validate(ff, ucell, ufw, scell, probe, dims, grid, None, 0.0, 0.0, [(pos - d) @ inv])
            fd_full.append((up[2] - dn[2]) / (2 * h))
        scale_t = max(1.0, np.abs(one[5:8]).max())
        scale_f = max(1.0, np.abs(one[8:11]).max())
        np.testing.assert_allclose(one[5:8], fd_table, rtol=0, atol=1e-5 * scale_t)
        np.testing.assert_allclose(one[8:11], fd_full, rtol=0, atol=1e-5 * scale_f)
    assert checked == 4


def test_oracle_triquintic_hessians_match_finite_differences(oracle):
    """The triquintic grid test's two Hessians (interpolated and analytical, xx, xy, xz, yy, yz, zz) are the central
    finite differences of its two gradients."""
    ff = synthetic_forcefield(charges=False)
    ucell, ufw = synthetic_framework(ff, seed=42)
    scell, _ = replicate(ucell, ufw, (2, 2, 3))
    dims = (21, 21, 14)
    probe = ff.index("CH4")
    grid = oracle.make_grid_triquintic(0, ff, ucell, ufw, probe, 12.0, dims)
    inv = np.linalg.inv(scell)
    rng = np.random.default_rng(12)
    h = 1e-5
    pairs = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]

    def values(pos):
        return oracle.grid_validate_triquintic(ff, ucell, ufw, scell, probe, dims, grid, None, 0.0, 0.0, [pos @ inv])

    checked = 0
    for _ in range(400):
        if checked == 3:
            break
        pos = rng.random(3) @ scell
        one = values(pos)
        if one[2] > 1e4:
            continue
        checked += 1
        up, dn = [], []
        for a in range(3):
            d = np.zeros(3)
            d[a] = h
            up.append(values(pos + d))
            dn.append(values(pos - d))
        for k, (i, j) in enumerate(pairs):
            fd_table = (up[j][5 + i] - dn[j][5 + i]) / (2 * h)
            fd_full = (up[j][8 + i] - dn[j][8 + i]) / (2 * h)
            scale_t = max(1.0, np.abs(one[36:42]).max())
            scale_f = max(1.0, np.abs(one[42:48]).max())
            assert abs(one[36 + k] - fd_table) < 1e-5 * scale_t, (k, one[36 + k], fd_table)
            assert abs(one[42 + k] - fd_full) < 1e-5 * scale_f, (k, one[42 + k], fd_full)
        # the energy and gradient parts agree with the interpolant and the analytical sum
        v, g = oracle.interpolate_triquintic(grid, dims, ucell, pos)
        assert one[1] == pytest.approx(v * ENERGY_TO_KELVIN, rel=1e-12)
        np.testing.assert_allclose(one[5:8], g * ENERGY_TO_KELVIN, rtol=1e-10, atol=1e-10)
    assert checked == 3

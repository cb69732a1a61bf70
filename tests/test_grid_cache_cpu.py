"""Grids on disk (host code, no GPU): the fingerprint of a grid's inputs, the binary cache round trip and its miss
cases, and the cube writer in the format of InterpolationEnergyGrid::writeOutput (interpolation_energy_grid.cpp:
4760-4789)."""

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ENERGY_TO_KELVIN
from raspa3_b200.synthetic import synthetic_forcefield, synthetic_framework

DIMS = (5, 4, 3)


@pytest.fixture(scope="module")
def system():
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    return ff, cell, atoms


def test_fingerprint_tracks_every_input(system):
    ff, cell, atoms = system
    probe = ff.index("CH4")
    base = native.grid_fingerprint(0, 8, ff, cell, atoms, probe, DIMS)
    assert base == native.grid_fingerprint(0, 8, ff, cell, atoms.copy(), probe, DIMS)
    moved = atoms.copy()
    moved["x"][7] += 1e-9
    charged = atoms.copy()
    charged["charge"][3] += 0.01
    variants = [
        native.grid_fingerprint(0, 8, ff, cell, moved, probe, DIMS),
        native.grid_fingerprint(0, 8, ff, cell, charged, probe, DIMS),
        native.grid_fingerprint(0, 8, ff, cell, atoms, ff.index("O_co2"), DIMS),
        native.grid_fingerprint(0, 8, ff, cell, atoms, probe, (5, 4, 4)),
        native.grid_fingerprint(0, 27, ff, cell, atoms, probe, DIMS),
        native.grid_fingerprint(0, 27, ff, cell, atoms, probe, DIMS, flags=1),
        native.grid_fingerprint(1, 8, ff, cell, atoms, probe, DIMS),
        native.grid_fingerprint(0, 8, ff, cell * 1.0001, atoms, probe, DIMS),
    ]
    ff2 = synthetic_forcefield(charges=True, rc=11.0)
    variants.append(native.grid_fingerprint(0, 8, ff2, cell, atoms, probe, DIMS))
    assert len(set(variants + [base])) == len(variants) + 1
    # the unit-charge Ewald grid does not depend on the probe
    assert native.grid_fingerprint(1, 8, ff, cell, atoms, probe, DIMS) == \
        native.grid_fingerprint(1, 8, ff, cell, atoms, ff.index("O_co2"), DIMS)


@pytest.mark.parametrize("scheme", [8, 27])
def test_save_load_round_trip_and_misses(system, tmp_path, oracle, scheme):
    ff, cell, atoms = system
    probe = ff.index("CH4")
    if scheme == 8:
        grid = oracle.make_grid(0, ff, cell, atoms, probe, 12.0, DIMS)
    else:
        grid = oracle.make_grid_triquintic(0, ff, cell, atoms, probe, 12.0, DIMS)
    key = native.grid_fingerprint(0, scheme, ff, cell, atoms, probe, DIMS)
    path = str(tmp_path / "ch4.grid")
    native.grid_save(path, key, scheme, cell, DIMS, grid)
    back = native.grid_load(path, key, scheme, DIMS)
    np.testing.assert_array_equal(back, grid)
    assert native.grid_load(path, key ^ 1, scheme, DIMS) is None          # other inputs
    assert native.grid_load(path, key, scheme, (5, 4, 4)) is None         # other shape
    assert native.grid_load(path, key, 35 - scheme, DIMS) is None         # other scheme
    assert native.grid_load(str(tmp_path / "none.grid"), key, scheme, DIMS) is None
    raw = bytearray(open(path, "rb").read())
    damaged = str(tmp_path / "damaged.grid")
    raw[-5] ^= 0x40
    open(damaged, "wb").write(raw)
    assert native.grid_load(damaged, key, scheme, DIMS) is None           # checksum
    open(damaged, "wb").write(bytes(raw[:len(raw) // 2]))
    assert native.grid_load(damaged, key, scheme, DIMS) is None           # truncated
    assert not (tmp_path / "ch4.grid.tmp").exists()


def test_cube_file_format(system, tmp_path, oracle):
    ff, cell, atoms = system
    grid = oracle.make_grid(0, ff, cell, atoms, ff.index("CH4"), 12.0, DIMS)
    path = str(tmp_path / "grid.cube")
    native.grid_write_cube(path, 8, grid, DIMS, cell, origin=[0.5, 0.0, -1.0])
    lines = open(path).read().splitlines()
    assert lines[0] == "Cube interpolation file" and lines[1] == "Written by RASPA-3"
    assert lines[2].split() == ["1", "0.5", "0", "-1"]
    for c in range(3):
        f = lines[3 + c].split()
        assert int(f[0]) == -DIMS[c]
        np.testing.assert_allclose([float(x) for x in f[1:]], cell[c] / DIMS[c], rtol=1e-15)
    assert lines[6] == "1 0.0 0.0 0.0 0.0"
    values = np.array([float(x) for x in lines[7:]])
    assert len(values) == np.prod(DIMS)
    # the energy channel in K, memory order (x fastest), shortest round-trip decimals
    np.testing.assert_array_equal(values, grid.reshape(-1, 8)[:, 0] * ENERGY_TO_KELVIN)

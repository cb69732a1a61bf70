"""The release-flag build of the oracle (the timed CPU baseline) computes the same grid values, trial energies and
Ewald energies as the strict build (the parity oracle), to the rounding that -ffast-math may reorder."""

import os
import subprocess
import sys

import pytest

SCRIPT = r"""
import sys, json
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
import oracle
from raspa3_b200.synthetic import synthetic_forcefield, synthetic_framework
from reference_systems import co2_atoms, itq29, zeolite_forcefield
if {release}:
    oracle.use_release_build()
ff = synthetic_forcefield(charges=True)
cell, atoms = synthetic_framework(ff)
pts = np.arange(0, 21 * 20 * 14, 7, dtype=np.int64)
g0 = oracle.make_grid(0, ff, cell, atoms, ff.index("C_co2"), 12.0, (21, 20, 14), points=pts)
g1 = oracle.make_grid(1, ff, cell, atoms, 0, 12.0, (21, 20, 14), points=pts)
ffz = zeolite_forcefield(12.0, True, use_charge=True)
ffz.ewald_alpha = 0.25
cz, fw = itq29(ffz)
c = 5.93355
mol = co2_atoms(ffz, [(c, 7.93355, c), (c, 3.93355, c)], [0, 1])
ok, e = oracle.cbmc_framework_molecule(ffz, cz, fw, mol, 12.0, 12.0)
ew, _ = oracle.ewald_fourier_energy(ffz, cz, mol, [3, 3], s_rigid=oracle.ewald_rigid(ffz, cz, fw))
print(json.dumps([g0.tolist(), g1.tolist(), [e["framework_molecule_vdw"], e["framework_molecule_charge"]],
                  [ew["ewald_fourier"], ew["ewald_self"], ew["ewald_exclusion"]]]))
"""


def run(release: bool):
    import json

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = SCRIPT.format(root=root, tests=os.path.join(root, "tests"), release=release)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_release_build_matches_strict_build():
    import numpy as np

    strict, release = run(False), run(True)
    for a, b in zip(strict, release):
        a, b = np.asarray(a), np.asarray(b)
        scale = np.maximum(np.abs(a), 1.0)
        assert np.all(np.abs(a - b) <= 1e-9 * scale), np.max(np.abs(a - b) / scale)

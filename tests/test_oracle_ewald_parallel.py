"""The all-cores CPU baseline of one Ewald Fourier difference (OpenMP over a precomputed k table) gives the serial
oracle's energy change and trial structure factors."""

import numpy as np

from raspa3_b200.synthetic import random_molecules, replicate, synthetic_forcefield, synthetic_framework


def test_parallel_delta_equals_serial(oracle):
    ff = synthetic_forcefield(charges=True, alpha=0.265, kmax=8)
    ucell, ufw = synthetic_framework(ff, seed=42)
    cell, _ = replicate(ucell, ufw, (2, 2, 3))
    ads = random_molecules(ff, cell, 30, seed=8)
    _, stored = oracle.ewald_fourier_energy(ff, cell, ads, np.full(30, 3, dtype=np.int32))
    par = oracle.EwaldDeltaParallel(ff, cell)
    rng = np.random.default_rng(3)
    for m in range(5):
        old = ads[3 * m:3 * m + 3].copy()
        new = old.copy()
        new["x"] += rng.normal()
        new["z"] -= rng.normal()
        ref, trial = oracle.ewald_delta(ff, cell, stored, new, old)
        t2 = np.zeros_like(stored)
        v = par(stored, new, old, t2)
        assert abs(v - ref["ewald_fourier"]) <= 1e-12 * max(1.0, abs(ref["ewald_fourier"]))
        np.testing.assert_allclose(t2.reshape(-1, 10)[:, :2], trial.reshape(-1, 10)[:, :2], rtol=0, atol=1e-12)

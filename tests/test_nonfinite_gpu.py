"""Failure detection on the host side of the C-ABI: a NaN or infinite position, charge or scaling factor in the input
is reported as RG_ERR_NONFINITE before anything is launched, and the context stays usable afterwards. The reference
has no such check (its sums would turn NaN). The faults are injected on the host."""

import ctypes

import numpy as np
import pytest

from raspa3_b200 import native
from raspa3_b200.forcefield import ATOM_DTYPE, box_struct, ff_struct
from raspa3_b200.synthetic import random_molecules, synthetic_forcefield, synthetic_framework

pytestmark = pytest.mark.gpu
RG_ERR_NONFINITE = 9


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def poisoned(atoms, field, index=0, value=float("nan")):
    a = atoms.copy()
    a[field][index] = value
    return a


def expect_nonfinite(fn):
    with pytest.raises(native.RaspaGpuError, match=f"status {RG_ERR_NONFINITE}"):
        fn()


@pytest.mark.parametrize("field,value", [("x", float("nan")), ("z", float("inf")), ("charge", float("nan"))])
def test_grid_builds_reject_nonfinite_atoms(ctx, field, value):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    bad = poisoned(atoms, field, 17, value)
    expect_nonfinite(lambda: ctx.grid_build(1, ff, cell, bad, 0, 12.0, (6, 6, 5)))
    expect_nonfinite(lambda: ctx.grid_build_triquintic(1, ff, cell, bad, 0, 12.0, (6, 6, 5)))
    torch = pytest.importorskip("torch")
    buf = torch.empty(8 * 6 * 6 * 5, dtype=torch.float64, device="cuda")
    expect_nonfinite(lambda: ctx.grid_build_set(ff, cell, bad, 12.0, (6, 6, 5), native.PRECISION_FP32C, [1], [0],
                                                [buf.data_ptr()]))
    a = np.ascontiguousarray(bad, dtype=ATOM_DTYPE)
    ffs, box = ff_struct(ff), box_struct(cell)
    st = native.lib().rg_grid_build_noalloc(0, None, 1, ctypes.byref(ffs), ctypes.byref(box),
                                            ctypes.c_void_p(a.ctypes.data), len(a), 0, 12.0, 6, 6, 5,
                                            native.PRECISION_FP64, ctypes.c_void_p(buf.data_ptr()), None)
    assert st == RG_ERR_NONFINITE
    # the context is still usable
    out, _ = ctx.grid_build(1, ff, cell, atoms, 0, 12.0, (6, 6, 5))
    assert np.all(np.isfinite(out))


def test_trial_energies_and_moves_reject_nonfinite_atoms(ctx):
    ff = synthetic_forcefield(charges=True)
    cell, atoms = synthetic_framework(ff)
    expect_nonfinite(lambda: native.System(ctx, ff, cell, poisoned(atoms, "y", 3)))
    sysg = native.System(ctx, ff, cell, atoms)
    try:
        ads = random_molecules(ff, cell, 4, seed=2)
        expect_nonfinite(lambda: sysg.set_molecules(poisoned(ads, "scaling_vdw", 5)))
        sysg.set_molecules(ads)
        expect_nonfinite(lambda: sysg.external_energies(poisoned(ads[:3], "x", 1), 3))
        expect_nonfinite(lambda: sysg.framework_energy_difference(poisoned(ads[:3], "z", 2, float("-inf")), ads[:3]))
        expect_nonfinite(lambda: sysg.intermolecular_energy_difference(ads[:3], poisoned(ads[:3], "charge", 0)))
        expect_nonfinite(lambda: sysg.update_molecules(0, poisoned(ads[:3], "scaling_coulomb", 1)))
        got = sysg.external_energies(ads[:3], 3)
        assert np.isfinite(got[0].framework_vdw)
        ew = native.Ewald(ctx, ff, cell)
        try:
            expect_nonfinite(lambda: ew.delta(poisoned(ads[:3], "x", 0), ads[:3]))
        finally:
            ew.close()
    finally:
        sysg.close()


def test_mixture_barrier_wait_gives_up_and_reports_timeout(ctx):
    """The bounded grid-barrier wait of the cooperative mixture kernel: with one CTA left out of the first barrier,
    every CTA's wait runs out after a short poll limit (no fault, no hang), rg_mixture_results reports RG_ERR_TIMEOUT,
    later launches do nothing, and the context stays usable for other work."""
    from raspa3_b200.forcefield import make_atoms
    from raspa3_b200.gcmc import beta_of, co2_component

    ff = synthetic_forcefield(charges=False)
    ff.cutoff_molecule_vdw = 1e-3
    L = 30.0
    empty = make_atoms(np.zeros((0, 3)), np.zeros(0, dtype=np.uint16), np.zeros(0))
    sysg = native.System(ctx, ff, np.diag([L, L, L]), empty)
    beta = beta_of(300.0)
    try:
        mx = native.Mixture(sysg, None, [co2_component()], beta, [3.0 / (beta * L ** 3)], np.zeros((0, 3, 3)),
                            np.zeros(0, dtype=np.int32), max_molecules=64, seed=3)
        try:
            mx.set_state(0.0)
            mx.run(200)
            ok = mx.results()
            assert ok["status"] == native.RG_OK and sum(ok["attempted"]) == 200
            mx.set_wait_test(1, 4096)
            mx.run(200)
            bad = mx.results()
            assert bad["status"] == 3  # RG_ERR_TIMEOUT
            assert bad["attempted"] == ok["attempted"]  # the failed launch made no move
            mx.set_wait_test(-1, 1 << 22)
            mx.run(200)  # the error flag persists: the launch returns at once
            again = mx.results()
            assert again["status"] == 3 and again["attempted"] == ok["attempted"]
            with pytest.raises(native.RaspaGpuError):
                mx.set_wait_test(10 ** 6, 100)
        finally:
            mx.close()
    finally:
        sysg.close()
    out, _ = ctx.grid_build(0, ff, np.diag([12.0, 12.0, 12.0]), empty, ff.index("CH4"), 12.0, (4, 4, 4))
    assert np.all(out == 0.0)

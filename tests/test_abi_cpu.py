"""CPU-only checks of the C-ABI library: it loads and exports every entry point include/raspa_gpu.h declares."""

import ctypes
import os
import re

import numpy as np

from raspa3_b200 import native
from raspa3_b200.forcefield import ATOM_DTYPE, RgForceField

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(rg_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    names = declared_functions()
    assert "rg_grid_build" in names and "rg_ctx_create" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string_without_device():
    assert b"sm_100a" in native.lib().rg_version()


def test_atom_record_matches_reference_layout():
    # src/raspakit/atom.ixx:28-39: double3 position (32 B), charge, scalingVDW, scalingCoulomb, u32, u16, u8, bits
    assert ATOM_DTYPE.itemsize == 64
    assert ATOM_DTYPE.fields["charge"][1] == 32
    assert ATOM_DTYPE.fields["molecule_id"][1] == 56
    assert ATOM_DTYPE.fields["type"][1] == 60
    assert ATOM_DTYPE.fields["group_fractional"][1] == 63
    assert ctypes.sizeof(RgForceField) == 4 + 4 + 8 * 4 + 8 * 4 + 12 + 4 + 8 + 8 + 8 + 4 + 4


def test_context_creation_without_device_reports_no_device():
    lib = native.lib()
    h = ctypes.c_void_p()
    st = lib.rg_ctx_create(0, ctypes.byref(h))
    # on a CPU-only machine there is no device; on a GPU machine creation succeeds
    if st == 0:
        lib.rg_ctx_destroy(h)
    else:
        assert st == 6  # RG_ERR_NO_DEVICE
    assert np.dtype(ATOM_DTYPE).names[0] == "x"

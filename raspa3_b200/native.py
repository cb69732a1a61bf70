"""ctypes binding of libraspagpu.so (the C-ABI declared in include/raspa_gpu.h).

The library is loaded from this package directory only; there is no fallback. If it is missing, or no CUDA device is
present, the calls raise — the GPU path never silently degrades to a CPU implementation.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .forcefield import ATOM_DTYPE, ForceField, RgBox, RgForceField, box_struct, ff_struct

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libraspagpu.so")

RG_OK = 0
GRID_LENNARD_JONES = 0
GRID_EWALD_REAL = 1
GRID_LENNARD_JONES_REPULSION = 2
GRID_LENNARD_JONES_ATTRACTION = 3
PRECISION_FP64 = 0
PRECISION_FP32C = 1

_lib = None


class RaspaGpuError(RuntimeError):
    pass


class GridStats(ctypes.Structure):
    _fields_ = [("pair_count", ctypes.c_int64), ("n_images", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RaspaGpuError(f"{LIB_PATH} is missing: build it with raspa3_b200.build.build() (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.rg_ctx_create.argtypes = [i32, P(vp)]
        L.rg_ctx_destroy.argtypes = [vp]
        L.rg_ctx_set_stream.argtypes = [vp, vp]
        L.rg_ctx_stream.argtypes = [vp]
        L.rg_ctx_stream.restype = vp
        L.rg_ctx_synchronize.argtypes = [vp]
        L.rg_ctx_last_error.argtypes = [vp]
        L.rg_ctx_last_error.restype = ctypes.c_char_p
        L.rg_version.restype = ctypes.c_char_p
        L.rg_grid_build.argtypes = [vp, i32, P(RgForceField), P(RgBox), vp, i32, i32, d, i32, i32, i32, i32, vp, vp,
                                    P(GridStats)]
        L.rg_probe_fma_peak.argtypes = [vp, i32, P(d), P(d)]
        _lib = L
    return _lib


def check(ctx_handle, status: int, what: str):
    if status != RG_OK:
        msg = lib().rg_ctx_last_error(ctx_handle).decode() if ctx_handle else ""
        raise RaspaGpuError(f"{what} failed with status {status}: {msg}")


class Context:
    """One rg_ctx: a device, a stream and grow-only scratch. Not shared between threads."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().rg_ctx_create(device, ctypes.byref(h))
        if st != RG_OK:
            raise RaspaGpuError(f"rg_ctx_create({device}) failed with status {st} (no CUDA device?)")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().rg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(self.handle, lib().rg_ctx_set_stream(self.handle, stream_ptr), "rg_ctx_set_stream")

    def synchronize(self):
        check(self.handle, lib().rg_ctx_synchronize(self.handle), "rg_ctx_synchronize")

    @property
    def stream(self) -> int:
        return lib().rg_ctx_stream(self.handle) or 0

    # ---- (a) grid build ----
    def grid_build(self, grid_type: int, ff: ForceField, cell, unit_atoms: np.ndarray, probe_type: int, cutoff: float,
                   dims, precision: int = PRECISION_FP64, out_device: int | None = None, host: bool = True,
                   count_pairs: bool = False, out_host: np.ndarray | None = None):
        """Returns (host array or None, stats dict or None). out_device: device pointer of 8*nx*ny*nz doubles;
        out_host: a caller-provided host float64 array (e.g. pinned) used instead of a fresh one."""
        nx, ny, nz = (int(v) for v in dims)
        atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
        ffs = ff_struct(ff)
        box = box_struct(cell)
        out = (out_host if out_host is not None else np.empty(8 * nx * ny * nz)) if host else None
        stats = GridStats()
        st = lib().rg_grid_build(self.handle, grid_type, ctypes.byref(ffs), ctypes.byref(box),
                                 ctypes.c_void_p(atoms.ctypes.data), len(atoms), probe_type, cutoff, nx, ny, nz,
                                 precision, out_device, None if out is None else ctypes.c_void_p(out.ctypes.data),
                                 ctypes.byref(stats) if count_pairs else None)
        check(self.handle, st, "rg_grid_build")
        return out, (stats.as_dict() if count_pairs else None)

    def probe_fma_peak(self, precision: int = PRECISION_FP32C) -> float:
        t, s = ctypes.c_double(), ctypes.c_double()
        check(self.handle, lib().rg_probe_fma_peak(self.handle, precision, ctypes.byref(t), ctypes.byref(s)),
              "rg_probe_fma_peak")
        return t.value

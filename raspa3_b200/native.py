"""ctypes binding of libraspagpu.so (the C-ABI declared in include/raspa_gpu.h).

The library is loaded from this package directory only; there is no fallback. If it is missing, or no CUDA device is
present, the calls raise — the GPU path never silently degrades to a CPU implementation.
"""

from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

from .forcefield import ATOM_DTYPE, ForceField, RgBox, RgForceField, box_struct, ff_struct

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libraspagpu.so")

RG_OK = 0
RG_ERR_CACHE_MISS = 8
GRID_LENNARD_JONES = 0
GRID_EWALD_REAL = 1
GRID_LENNARD_JONES_REPULSION = 2
GRID_LENNARD_JONES_ATTRACTION = 3
PRECISION_FP64 = 0
PRECISION_FP32C = 1
CHARGE_METHOD_EWALD = 0
CHARGE_METHOD_COULOMB = 1
SURFACE_OFF = -1
SURFACE_NONE = 0
SURFACE_GRID_FILE = 1
SURFACE_THIRD_ORDER_POLYNOMIAL = 3
SURFACE_MULLER_BROWN = 8
SURFACE_CYLINDER_X = 11
SURFACE_CYLINDER_Y = 12
SURFACE_CYLINDER_Z = 13
SURFACE_RECTANGLE_X = 14
SURFACE_RECTANGLE_Y = 15
SURFACE_RECTANGLE_Z = 16
SCHEME_TRICUBIC = 8
SCHEME_TRIQUINTIC = 27
TRIQUINTIC_REFERENCE_RECTANGULAR = 1
TRIQUINTIC_FP32C = 2

_lib = None


class RaspaGpuError(RuntimeError):
    pass


class EwaldEnergy(ctypes.Structure):
    _fields_ = [("ewald_fourier", ctypes.c_double), ("ewald_self", ctypes.c_double),
                ("ewald_exclusion", ctypes.c_double), ("dudlambda_ewald", ctypes.c_double * 4)]

    def as_dict(self):
        return {"ewald_fourier": self.ewald_fourier, "ewald_self": self.ewald_self,
                "ewald_exclusion": self.ewald_exclusion, "dudlambda_ewald": list(self.dudlambda_ewald)}


class TrialEnergy(ctypes.Structure):
    _fields_ = [("framework_vdw", ctypes.c_double), ("framework_charge", ctypes.c_double),
                ("molecule_vdw", ctypes.c_double), ("molecule_charge", ctypes.c_double),
                ("dudlambda_vdw", ctypes.c_double * 4), ("dudlambda_charge", ctypes.c_double * 4),
                ("external_field_vdw", ctypes.c_double), ("overlap", ctypes.c_int32), ("pad", ctypes.c_int32)]


class GcmcComponent(ctypes.Structure):
    _fields_ = [("n_atoms", ctypes.c_int32), ("starting_bead", ctypes.c_int32), ("types", ctypes.c_int32 * 8),
                ("charges", ctypes.c_double * 8), ("masses", ctypes.c_double * 8), ("offsets", ctypes.c_double * 24)]


class GcmcParams(ctypes.Structure):
    _fields_ = [("beta", ctypes.c_double), ("fugacity", ctypes.c_double),
                ("cutoff_framework_vdw", ctypes.c_double), ("cutoff_molecule_vdw", ctypes.c_double),
                ("cutoff_coulomb", ctypes.c_double), ("max_translation", ctypes.c_double),
                ("max_rotation", ctypes.c_double), ("p_translation", ctypes.c_double),
                ("p_rotation", ctypes.c_double), ("p_swap", ctypes.c_double),
                ("n_first_bead_trials", ctypes.c_int32), ("n_orientation_trials", ctypes.c_int32),
                ("max_molecules", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class GcmcChainResult(ctypes.Structure):
    _fields_ = [("n_molecules", ctypes.c_int64), ("energy", ctypes.c_double), ("attempted", ctypes.c_int64 * 4),
                ("accepted", ctypes.c_int64 * 4), ("sum_n", ctypes.c_double), ("sum_n2", ctypes.c_double),
                ("sum_energy", ctypes.c_double), ("samples", ctypes.c_int64), ("block_n", ctypes.c_double * 5)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("attempted", "accepted", "block_n")}
        d["attempted"], d["accepted"], d["block_n"] = list(self.attempted), list(self.accepted), list(self.block_n)
        return d


class MixtureParams(ctypes.Structure):
    _fields_ = [("beta", ctypes.c_double), ("fugacity", ctypes.c_double * 4), ("w_ig", ctypes.c_double * 4),
                ("cutoff_molecule_vdw", ctypes.c_double), ("cutoff_coulomb", ctypes.c_double),
                ("cutoff_framework_vdw", ctypes.c_double), ("max_translation", ctypes.c_double), ("max_rotation", ctypes.c_double),
                ("p_translation", ctypes.c_double), ("p_rotation", ctypes.c_double), ("p_swap", ctypes.c_double),
                ("p_identity", ctypes.c_double), ("n_first_bead_trials", ctypes.c_int32),
                ("n_orientation_trials", ctypes.c_int32), ("max_molecules", ctypes.c_int32),
                ("n_blocks", ctypes.c_int32), ("seed", ctypes.c_uint64)]


class MixtureResult(ctypes.Structure):
    _fields_ = [("n_molecules", ctypes.c_int64 * 4), ("energy", ctypes.c_double), ("attempted", ctypes.c_int64 * 5),
                ("accepted", ctypes.c_int64 * 5), ("sum_n", ctypes.c_double * 4), ("sum_energy", ctypes.c_double),
                ("samples", ctypes.c_int64), ("status", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    def as_dict(self):
        return {"n_molecules": list(self.n_molecules), "energy": self.energy, "attempted": list(self.attempted),
                "accepted": list(self.accepted), "sum_n": list(self.sum_n), "sum_energy": self.sum_energy,
                "samples": self.samples, "status": self.status}


class AlkanePlan(ctypes.Structure):
    _fields_ = [("cluster_big", ctypes.c_int32), ("cluster_small", ctypes.c_int32), ("threads", ctypes.c_int32),
                ("split", ctypes.c_int32), ("moves_per_launch", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("ms_per_move", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class GridStats(ctypes.Structure):
    _fields_ = [("pair_count", ctypes.c_int64), ("n_images", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64),
                ("d2h_bytes", ctypes.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class GridValidation(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int64), ("n_points_charge", ctypes.c_int64), ("sums", ctypes.c_double * 34),
                ("energy_table", ctypes.c_double), ("energy_full", ctypes.c_double),
                ("energy_relative_error", ctypes.c_double), ("gradient_table", ctypes.c_double * 3),
                ("gradient_full", ctypes.c_double * 3), ("gradient_relative_error", ctypes.c_double * 3),
                ("charge_energy_table", ctypes.c_double), ("charge_energy_full", ctypes.c_double),
                ("charge_energy_relative_error", ctypes.c_double), ("charge_gradient_table", ctypes.c_double * 3),
                ("charge_gradient_full", ctypes.c_double * 3), ("charge_gradient_relative_error", ctypes.c_double * 3)]

    def as_dict(self):
        out = {}
        for f, _ in self._fields_:
            v = getattr(self, f)
            out[f] = list(v) if isinstance(v, ctypes.Array) else v
        return out


class GridValidationHessian(ctypes.Structure):
    _fields_ = [("sums", ctypes.c_double * 48), ("hessian_table", ctypes.c_double * 6),
                ("hessian_full", ctypes.c_double * 6), ("hessian_relative_error", ctypes.c_double * 6),
                ("charge_hessian_table", ctypes.c_double * 6), ("charge_hessian_full", ctypes.c_double * 6),
                ("charge_hessian_relative_error", ctypes.c_double * 6)]

    def as_dict(self):
        return {f: list(getattr(self, f)) for f, _ in self._fields_}


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
        L.rg_grid_build_triquintic.argtypes = [vp, i32, P(RgForceField), P(RgBox), vp, i32, i32, d, i32, i32, i32, i32,
                                               vp, vp, P(GridStats)]
        L.rg_grid_interpolate.argtypes = [vp, i32, vp, i32, i32, i32, P(RgBox), vp, i32, vp, vp]
        L.rg_grid_fingerprint.argtypes = [i32, i32, i32, P(RgForceField), P(RgBox), vp, i32, i32, i32, i32, i32]
        L.rg_grid_fingerprint.restype = ctypes.c_uint64
        L.rg_grid_save.argtypes = [ctypes.c_char_p, ctypes.c_uint64, i32, P(RgBox), i32, i32, i32, vp]
        L.rg_grid_load.argtypes = [ctypes.c_char_p, ctypes.c_uint64, i32, i32, i32, i32, vp]
        L.rg_grid_write_cube.argtypes = [ctypes.c_char_p, i32, vp, i32, i32, i32, P(RgBox), vp]
        L.rg_grid_build_set.argtypes = [vp, P(RgForceField), P(RgBox), vp, i32, d, i32, i32, i32, i32, i32, vp, vp, vp,
                                        vp, vp]
        L.rg_grid_validate.argtypes = [vp, P(RgForceField), P(RgBox), vp, i32, P(RgBox), i32, i32, i32, i32, vp, vp, d,
                                       d, i64, ctypes.c_uint64, vp, P(GridValidation)]
        L.rg_grid_validate_triquintic.argtypes = [vp, P(RgForceField), P(RgBox), vp, i32, P(RgBox), i32, i32, i32, i32,
                                                  vp, vp, d, d, i64, ctypes.c_uint64, vp, P(GridValidation),
                                                  P(GridValidationHessian)]
        L.rg_grid_build_noalloc.argtypes = [i32, vp, i32, P(RgForceField), P(RgBox), vp, i32, i32, d, i32, i32, i32,
                                            i32, vp, P(GridStats)]
        L.rg_system_create.argtypes = [vp, P(RgForceField), P(RgBox), vp, i32, P(vp)]
        L.rg_system_destroy.argtypes = [vp]
        L.rg_system_set_grid.argtypes = [vp, i32, P(RgBox), i32, i32, i32, vp, i32]
        L.rg_system_set_interpolation_scheme.argtypes = [vp, i32]
        L.rg_system_set_molecules.argtypes = [vp, vp, i32]
        L.rg_system_set_precision.argtypes = [vp, i32]
        L.rg_cbmc_external_energies.argtypes = [vp, vp, i32, i32, i32, i64, d, d, d, vp]
        L.rg_cbmc_dual_cutoff_correction.argtypes = [vp, vp, i32, i64, d, vp]
        L.rg_framework_molecule_energy_difference.argtypes = [vp, i32, vp, i32, vp, i32, vp]
        L.rg_intermolecular_energy_difference.argtypes = [vp, vp, i32, vp, i32, vp]
        L.rg_system_update_molecules.argtypes = [vp, i32, vp, i32]
        L.rg_system_set_blocked_pockets.argtypes = [vp, P(RgBox), vp, i32]
        L.rg_system_set_external_field.argtypes = [vp, i32, vp, P(RgBox), i32, i32, i32, vp, i32]
        L.rg_gcmc_create.argtypes = [vp, vp, P(GcmcComponent), P(GcmcParams), i32, P(vp)]
        L.rg_gcmc_destroy.argtypes = [vp]
        L.rg_gcmc_run.argtypes = [vp, i64, i32]
        L.rg_gcmc_results.argtypes = [vp, vp]
        L.rg_gcmc_get_positions.argtypes = [vp, i32, vp, i32, P(i32)]
        L.rg_gcmc_set_proposal.argtypes = [vp, vp, P(RgBox)]
        L.rg_mlp_create.argtypes = [vp, ctypes.c_uint64, P(vp)]
        L.rg_mlp_destroy.argtypes = [vp]
        L.rg_mlp_num_params.restype = i32
        L.rg_mlp_get_params.argtypes = [vp, vp, i32]
        L.rg_mlp_set_params.argtypes = [vp, vp, i32]
        L.rg_mlp_loss_and_gradient.argtypes = [vp, vp, vp, i32, P(ctypes.c_float), vp]
        L.rg_mlp_train.argtypes = [vp, vp, vp, i64, i32, i32, ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)]
        L.rg_mlp_evaluate.argtypes = [vp, vp, i64, vp]
        L.rg_proposal_sample_targets.argtypes = [vp, i32, d, d, d, P(RgBox), i64, ctypes.c_uint64, vp, vp]
        L.rg_proposal_create.argtypes = [vp, i32, d, P(vp)]
        L.rg_proposal_destroy.argtypes = [vp]
        L.rg_proposal_density.argtypes = [vp, vp, i64, vp]
        L.rg_ewald_create.argtypes = [vp, P(RgForceField), P(RgBox), i32, P(vp)]
        L.rg_ewald_destroy.argtypes = [vp]
        L.rg_ewald_info.argtypes = [vp, P(i64), P(d)]
        L.rg_ewald_set_framework.argtypes = [vp, vp, i32]
        L.rg_ewald_full.argtypes = [vp, vp, i32, vp, i32, d, P(EwaldEnergy)]
        L.rg_ewald_delta.argtypes = [vp, vp, i32, vp, i32, d, vp, P(EwaldEnergy)]
        L.rg_ewald_accept.argtypes = [vp]
        L.rg_ewald_get_structure_factors.argtypes = [vp, i32, vp, i64]
        L.rg_ewald_set_structure_factors.argtypes = [vp, vp, i64]
        L.rg_mixture_create.argtypes = [vp, vp, vp, i32, P(MixtureParams), vp, vp, i32, P(vp)]
        L.rg_mixture_destroy.argtypes = [vp]
        L.rg_mixture_set_state.argtypes = [vp, d, vp, i64]
        L.rg_mixture_run.argtypes = [vp, i64, i32]
        L.rg_mixture_results.argtypes = [vp, P(MixtureResult)]
        L.rg_mixture_set_wait_test.argtypes = [vp, i32, i64]
        L.rg_mixture_run_many.argtypes = [vp, i32, i64, i32]
        L.rg_ewald_batch_create.argtypes = [vp, i32, P(vp)]
        L.rg_ewald_batch_destroy.argtypes = [vp]
        L.rg_ewald_batch_set.argtypes = [vp, i32, vp]
        L.rg_ewald_batch_get.argtypes = [vp, i32, i32, vp]
        L.rg_ewald_batch_delta.argtypes = [vp, vp, i32, vp, vp, vp]
        L.rg_ewald_batch_accept.argtypes = [vp, vp]
        L.rg_ewald_batch_timing.argtypes = [vp, P(ctypes.c_float), P(ctypes.c_float)]
        L.rg_mixture_get_positions.argtypes = [vp, vp, vp, i32, P(i32)]
        L.rg_mixture_get_structure_factors.argtypes = [vp, vp, i64]
        L.rg_mixture_set_proposal.argtypes = [vp, i32, vp, P(RgBox)]
        L.rg_mixture_info.argtypes = [vp, P(i32), P(i64)]
        from .alkane import RgAlkaneChain
        L.rg_alkane_create.argtypes = [vp, P(RgForceField), vp, i32, ctypes.c_uint64, P(vp)]
        L.rg_alkane_destroy.argtypes = [vp]
        L.rg_alkane_autotune.argtypes = [vp, i32, P(AlkanePlan)]
        L.rg_alkane_set_plan.argtypes = [vp, P(AlkanePlan)]
        L.rg_alkane_get_plan.argtypes = [vp, P(AlkanePlan)]
        L.rg_alkane_run.argtypes = [vp, i64, i32]
        L.rg_alkane_results.argtypes = [vp, vp]
        L.rg_alkane_get_positions.argtypes = [vp, i32, vp, i32, P(i32)]
        L.rg_alkane_set_positions.argtypes = [vp, i32, vp, i32, d]
        L.rg_alkane_pair_count.argtypes = [vp, P(ctypes.c_uint64)]
        L.rg_alkane_launch_count.argtypes = [vp, P(ctypes.c_int64)]
        L.rg_alkane_bead_energies.argtypes = [vp, i32, vp, vp, i32, i32, vp, vp, vp]
        L.rg_alkane_grow_vacuum.argtypes = [vp, P(RgForceField), P(RgAlkaneChain), d, i64, ctypes.c_uint64, P(d), vp,
                                            vp, vp]
        _lib = L
    return _lib


def check(ctx_handle, status: int, what: str):
    if status != RG_OK:
        msg = lib().rg_ctx_last_error(ctx_handle).decode() if ctx_handle else ""
        raise RaspaGpuError(f"{what} failed with status {status}: {msg}")


def grid_fingerprint(grid_type: int, scheme: int, ff: ForceField, cell, unit_atoms, probe_type: int, dims,
                     flags: int = 0) -> int:
    """rg_grid_fingerprint: 64-bit key of every input that determines a grid."""
    atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
    ffs, box = ff_struct(ff), box_struct(cell)
    return int(lib().rg_grid_fingerprint(grid_type, scheme, flags, ctypes.byref(ffs), ctypes.byref(box),
                                         ctypes.c_void_p(atoms.ctypes.data), len(atoms), probe_type, *dims))


def grid_save(path: str, fingerprint: int, scheme: int, cell, dims, data: np.ndarray):
    d = np.ascontiguousarray(data, dtype=np.float64)
    st = lib().rg_grid_save(path.encode(), fingerprint, scheme, ctypes.byref(box_struct(cell)), *dims,
                            ctypes.c_void_p(d.ctypes.data))
    check(None, st, "rg_grid_save")


def grid_load(path: str, fingerprint: int, scheme: int, dims):
    """The cached grid, or None on a cache miss (no file, other inputs or shape, damaged file)."""
    out = np.empty(scheme * int(np.prod(dims)))
    st = lib().rg_grid_load(path.encode(), fingerprint, scheme, *dims, ctypes.c_void_p(out.ctypes.data))
    if st == RG_ERR_CACHE_MISS:
        return None
    check(None, st, "rg_grid_load")
    return out


def grid_write_cube(path: str, scheme: int, data: np.ndarray, dims, cell, origin=None):
    d = np.ascontiguousarray(data, dtype=np.float64)
    o = None if origin is None else np.ascontiguousarray(origin, dtype=np.float64)
    st = lib().rg_grid_write_cube(path.encode(), scheme, ctypes.c_void_p(d.ctypes.data), *dims,
                                  ctypes.byref(box_struct(cell)), None if o is None else ctypes.c_void_p(o.ctypes.data))
    check(None, st, "rg_grid_write_cube")


class Context:
    """One rg_ctx: a device, a stream and grow-only scratch. Not shared between threads."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().rg_ctx_create(device, ctypes.byref(h))
        if st != RG_OK:
            raise RaspaGpuError(f"rg_ctx_create({device}) failed with status {st} (no CUDA device?)")
        self.handle = h
        self.device = device
        self._children = weakref.WeakSet()

    def adopt(self, child):
        """Objects created on this context (systems, Ewald states, GCMC runs) are closed before it."""
        self._children.add(child)

    def close(self):
        if self.handle:
            for child in list(self._children):
                child.close()
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

    def grid_build_triquintic(self, grid_type: int, ff: ForceField, cell, unit_atoms: np.ndarray, probe_type: int,
                              cutoff: float, dims, reference_rectangular: bool = False, out_device: int | None = None,
                              host: bool = True, count_pairs: bool = False, out_host: np.ndarray | None = None,
                              fp32c: bool = False):
        """Triquintic grid (27 doubles per point, rg_grid_build_triquintic). Returns (host array or None, stats or
        None); out_device: device pointer of 27*nx*ny*nz doubles; out_host: a caller-provided host float64 array
        (e.g. pinned) used instead of a fresh one."""
        nx, ny, nz = (int(v) for v in dims)
        atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
        ffs, box = ff_struct(ff), box_struct(cell)
        out = (out_host if out_host is not None else np.empty(27 * nx * ny * nz)) if host else None
        stats = GridStats()
        flags = (TRIQUINTIC_REFERENCE_RECTANGULAR if reference_rectangular else 0) | (TRIQUINTIC_FP32C if fp32c else 0)
        st = lib().rg_grid_build_triquintic(self.handle, grid_type, ctypes.byref(ffs), ctypes.byref(box),
                                            ctypes.c_void_p(atoms.ctypes.data), len(atoms), probe_type, cutoff, nx, ny,
                                            nz, flags, out_device,
                                            None if out is None else ctypes.c_void_p(out.ctypes.data),
                                            ctypes.byref(stats) if count_pairs else None)
        check(self.handle, st, "rg_grid_build_triquintic")
        return out, (stats.as_dict() if count_pairs else None)

    def grid_interpolate(self, scheme: int, grid_device: int, dims, cell, positions, gradients: bool = True):
        """Values (and Cartesian gradients) of a device grid at Cartesian positions (rg_grid_interpolate)."""
        nx, ny, nz = (int(v) for v in dims)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        e = np.empty(n)
        g = np.empty((n, 3)) if gradients else None
        box = box_struct(cell)
        st = lib().rg_grid_interpolate(self.handle, scheme, ctypes.c_void_p(grid_device), nx, ny, nz,
                                       ctypes.byref(box), ctypes.c_void_p(pos.ctypes.data), n,
                                       ctypes.c_void_p(e.ctypes.data),
                                       None if g is None else ctypes.c_void_p(g.ctypes.data))
        check(self.handle, st, "rg_grid_interpolate")
        return e, g

    def grid_validate(self, ff: ForceField, unit_cell, unit_atoms: np.ndarray, simulation_cell, probe_type: int, dims,
                      vdw_grid_device: int, ewald_grid_device: int | None = None, probe_charge: float = 0.0,
                      weight_beta: float = 1.0 / 300.0, n_points: int = 100000, seed: int = 1, points=None) -> dict:
        """The reference's grid test on the device (rg_grid_validate): Boltzmann-weighted sums, averages and relative
        errors of the interpolated vs analytical energy and gradient. points: (n, 3) fractions of the simulation box,
        or None for n_points Philox points from seed."""
        nx, ny, nz = (int(v) for v in dims)
        atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
        pts = None if points is None else np.ascontiguousarray(points, dtype=np.float64)
        n = n_points if pts is None else len(pts)
        out = GridValidation()
        ffs, ubox, sbox = ff_struct(ff), box_struct(unit_cell), box_struct(simulation_cell)
        st = lib().rg_grid_validate(self.handle, ctypes.byref(ffs), ctypes.byref(ubox),
                                    ctypes.c_void_p(atoms.ctypes.data), len(atoms), ctypes.byref(sbox), probe_type,
                                    nx, ny, nz,
                                    ctypes.c_void_p(vdw_grid_device),
                                    ctypes.c_void_p(ewald_grid_device) if ewald_grid_device else None, probe_charge,
                                    weight_beta, n, seed, ctypes.c_void_p(pts.ctypes.data) if pts is not None else None,
                                    ctypes.byref(out))
        check(self.handle, st, "rg_grid_validate")
        return out.as_dict()

    def grid_validate_triquintic(self, ff: ForceField, unit_cell, unit_atoms: np.ndarray, simulation_cell,
                                 probe_type: int, dims, vdw_grid_device: int, ewald_grid_device: int | None = None,
                                 probe_charge: float = 0.0, weight_beta: float = 1.0 / 300.0, n_points: int = 100000,
                                 seed: int = 1, points=None):
        """The triquintic grid test (rg_grid_validate_triquintic): the dict of grid_validate plus a "hessian" dict."""
        nx, ny, nz = (int(v) for v in dims)
        atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
        pts = None if points is None else np.ascontiguousarray(points, dtype=np.float64)
        n = n_points if pts is None else len(pts)
        out, hess = GridValidation(), GridValidationHessian()
        ffs, ubox, sbox = ff_struct(ff), box_struct(unit_cell), box_struct(simulation_cell)
        st = lib().rg_grid_validate_triquintic(
            self.handle, ctypes.byref(ffs), ctypes.byref(ubox), ctypes.c_void_p(atoms.ctypes.data), len(atoms),
            ctypes.byref(sbox), probe_type, nx, ny, nz, ctypes.c_void_p(vdw_grid_device),
            ctypes.c_void_p(ewald_grid_device) if ewald_grid_device else None, probe_charge, weight_beta, n, seed,
            ctypes.c_void_p(pts.ctypes.data) if pts is not None else None, ctypes.byref(out), ctypes.byref(hess))
        check(self.handle, st, "rg_grid_validate_triquintic")
        d = out.as_dict()
        d["hessian"] = hess.as_dict()
        return d

    def grid_build_set(self, ff: ForceField, cell, unit_atoms: np.ndarray, cutoff: float, dims, precision: int,
                       grid_types, probe_types, out_device_ptrs, count_pairs: bool = False, out_host=None):
        """Several grids of one framework into device buffers (Lennard-Jones probes fused in pairs); out_host: optional
        list of host float64 arrays that also receive the grids."""
        nx, ny, nz = (int(v) for v in dims)
        atoms = np.ascontiguousarray(unit_atoms, dtype=ATOM_DTYPE)
        ffs, box = ff_struct(ff), box_struct(cell)
        n = len(grid_types)
        gt = np.ascontiguousarray(grid_types, dtype=np.int32)
        pt = np.ascontiguousarray(probe_types, dtype=np.int32)
        outs = (ctypes.c_void_p * n)(*[int(p) for p in out_device_ptrs])
        hosts = None
        if out_host is not None:
            hosts = (ctypes.c_void_p * n)(*[None if h is None else h.ctypes.data for h in out_host])
        stats = (GridStats * n)()
        check(self.handle, lib().rg_grid_build_set(self.handle, ctypes.byref(ffs), ctypes.byref(box),
                                                   ctypes.c_void_p(atoms.ctypes.data), len(atoms), cutoff, nx, ny, nz,
                                                   precision, n, ctypes.c_void_p(gt.ctypes.data),
                                                   ctypes.c_void_p(pt.ctypes.data), ctypes.cast(outs, ctypes.c_void_p),
                                                   None if hosts is None else ctypes.cast(hosts, ctypes.c_void_p),
                                                   ctypes.cast(stats, ctypes.c_void_p) if count_pairs else None),
              "rg_grid_build_set")
        return [stats[i].as_dict() for i in range(n)] if count_pairs else None

    def probe_fma_peak(self, precision: int = PRECISION_FP32C) -> float:
        t, s = ctypes.c_double(), ctypes.c_double()
        check(self.handle, lib().rg_probe_fma_peak(self.handle, precision, ctypes.byref(t), ctypes.byref(s)),
              "rg_probe_fma_peak")
        return t.value


def _atoms_ptr(a):
    if not (isinstance(a, np.ndarray) and a.dtype == ATOM_DTYPE and a.flags.c_contiguous):
        a = np.ascontiguousarray(a, dtype=ATOM_DTYPE)
    return a, (a.ctypes.data if len(a) else None)


def _ewald_delta(*args):
    global _ewald_delta_fn
    if _ewald_delta_fn is None:
        _ewald_delta_fn = lib().rg_ewald_delta
    return _ewald_delta_fn(*args)


_ewald_delta_fn = None


class Ewald:
    """Device-resident Ewald state of one system (k-vectors, prefactors, stored/trial structure factors)."""

    def __init__(self, ctx: Context, ff: ForceField, cell, n_groups: int = 0):
        self.ctx = ctx
        self._ff = ff_struct(ff)
        self._box = box_struct(cell)
        h = ctypes.c_void_p()
        check(ctx.handle, lib().rg_ewald_create(ctx.handle, ctypes.byref(self._ff), ctypes.byref(self._box), n_groups,
                                                ctypes.byref(h)), "rg_ewald_create")
        self.handle = h
        ctx.adopt(self)
        self.n_groups = n_groups
        nk, s = ctypes.c_int64(), ctypes.c_double()
        check(ctx.handle, lib().rg_ewald_info(h, ctypes.byref(nk), ctypes.byref(s)), "rg_ewald_info")
        self.n_kvectors = nk.value
        self.single_ion_sum = s.value

    def close(self):
        if self.handle:
            lib().rg_ewald_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_framework(self, fw_atoms):
        a, p = _atoms_ptr(fw_atoms)
        check(self.ctx.handle, lib().rg_ewald_set_framework(self.handle, p, len(a)), "rg_ewald_set_framework")

    def full(self, atoms, molecule_sizes, net_charge_framework=0.0) -> dict:
        a, p = _atoms_ptr(atoms)
        ms = np.ascontiguousarray(molecule_sizes, dtype=np.int32)
        e = EwaldEnergy()
        check(self.ctx.handle, lib().rg_ewald_full(self.handle, p, len(a), ctypes.c_void_p(ms.ctypes.data) if len(ms)
                                                   else None, len(ms), net_charge_framework, ctypes.byref(e)),
              "rg_ewald_full")
        return e.as_dict()

    def delta(self, new_atoms, old_atoms, net_charge=0.0, net_charge_derivative_ext=None) -> dict:
        na, pn = _atoms_ptr(new_atoms)
        oa, po = _atoms_ptr(old_atoms)
        nd = None
        if net_charge_derivative_ext is not None:
            nd = np.ascontiguousarray(net_charge_derivative_ext, dtype=np.float64)
        e = EwaldEnergy()
        st = _ewald_delta(self.handle, pn, len(na), po, len(oa), net_charge, None if nd is None else nd.ctypes.data,
                          ctypes.byref(e))
        if st:
            check(self.ctx.handle, st, "rg_ewald_delta")
        return e.as_dict()

    def accept(self):
        check(self.ctx.handle, lib().rg_ewald_accept(self.handle), "rg_ewald_accept")

    def structure_factors(self, which: int = 0) -> np.ndarray:
        n = 2 * self.n_kvectors * (1 + self.n_groups)
        out = np.empty(n)
        check(self.ctx.handle, lib().rg_ewald_get_structure_factors(self.handle, which, ctypes.c_void_p(out.ctypes.data),
                                                                    n), "rg_ewald_get_structure_factors")
        return out if which != 2 else out[: 2 * self.n_kvectors]

    def set_structure_factors(self, s: np.ndarray):
        s = np.ascontiguousarray(s, dtype=np.float64)
        check(self.ctx.handle, lib().rg_ewald_set_structure_factors(self.handle, ctypes.c_void_p(s.ctypes.data),
                                                                    len(s)), "rg_ewald_set_structure_factors")


class System:
    """Device-resident framework, grids and adsorbates of one system (the CBMC::GrowContext data)."""

    def __init__(self, ctx: Context, ff: ForceField, cell, framework_atoms):
        self.ctx = ctx
        self.ff = ff
        self._ff = ff_struct(ff)
        self._box = box_struct(cell)
        fw, p = _atoms_ptr(framework_atoms)
        self._fw = fw
        h = ctypes.c_void_p()
        check(ctx.handle, lib().rg_system_create(ctx.handle, ctypes.byref(self._ff), ctypes.byref(self._box), p,
                                                 len(fw), ctypes.byref(h)), "rg_system_create")
        self.handle = h
        ctx.adopt(self)
        self._grids = {}

    def close(self):
        if self.handle:
            lib().rg_system_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_grid(self, index: int, unit_cell, dims, data, on_device: bool = False):
        box = box_struct(unit_cell)
        if on_device:
            ptr = ctypes.c_void_p(int(data))
        else:
            data = np.ascontiguousarray(data, dtype=np.float64)
            self._grids[index] = data
            ptr = ctypes.c_void_p(data.ctypes.data)
        check(self.ctx.handle, lib().rg_system_set_grid(self.handle, index, ctypes.byref(box), dims[0], dims[1],
                                                        dims[2], ptr, 1 if on_device else 0), "rg_system_set_grid")

    def set_molecules(self, atoms):
        a, p = _atoms_ptr(atoms)
        check(self.ctx.handle, lib().rg_system_set_molecules(self.handle, p, len(a)), "rg_system_set_molecules")

    def set_interpolation_scheme(self, scheme: int):
        check(self.ctx.handle, lib().rg_system_set_interpolation_scheme(self.handle, scheme),
              "rg_system_set_interpolation_scheme")

    def set_precision(self, precision: int):
        """Arithmetic of external_energies: PRECISION_FP64 (default) or PRECISION_FP32C."""
        check(self.ctx.handle, lib().rg_system_set_precision(self.handle, precision), "rg_system_set_precision")

    def external_energies(self, trials, atoms_per_trial: int, skip: int = -1, skip_background: int = -1,
                          cutoff_framework_vdw: float | None = None, cutoff_molecule_vdw: float | None = None,
                          cutoff_coulomb: float | None = None):
        t, p = _atoms_ptr(trials)
        n = len(t) // atoms_per_trial
        out = (TrialEnergy * max(n, 1))()
        ff = self.ff
        check(self.ctx.handle, lib().rg_cbmc_external_energies(
            self.handle, p, n, atoms_per_trial, skip, skip_background,
            ff.cutoff_framework_vdw if cutoff_framework_vdw is None else cutoff_framework_vdw,
            ff.cutoff_molecule_vdw if cutoff_molecule_vdw is None else cutoff_molecule_vdw,
            ff.cutoff_coulomb if cutoff_coulomb is None else cutoff_coulomb, ctypes.cast(out, ctypes.c_void_p)),
            "rg_cbmc_external_energies")
        return [out[i] for i in range(n)]

    def dual_cutoff_correction(self, trial_set, dual_cutoff: float, skip_background: int = -1) -> TrialEnergy:
        """CBMC::computeDualCutOffCorrection of one trial set (rg_cbmc_dual_cutoff_correction)."""
        t, p = _atoms_ptr(trial_set)
        out = TrialEnergy()
        check(self.ctx.handle, lib().rg_cbmc_dual_cutoff_correction(self.handle, p, len(t), skip_background,
                                                                     dual_cutoff, ctypes.byref(out)),
              "rg_cbmc_dual_cutoff_correction")
        return out

    def framework_energy_difference(self, new_atoms, old_atoms, charge_method: int = CHARGE_METHOD_EWALD):
        """Interactions::computeFrameworkMoleculeEnergyDifference (rg_framework_molecule_energy_difference)."""
        n, pn = _atoms_ptr(new_atoms)
        o, po = _atoms_ptr(old_atoms)
        out = TrialEnergy()
        check(self.ctx.handle, lib().rg_framework_molecule_energy_difference(self.handle, charge_method, pn, len(n), po,
                                                                              len(o), ctypes.byref(out)),
              "rg_framework_molecule_energy_difference")
        return out

    def intermolecular_energy_difference(self, new_atoms, old_atoms):
        """Interactions::computeInterMolecularEnergyDifference (rg_intermolecular_energy_difference)."""
        n, pn = _atoms_ptr(new_atoms)
        o, po = _atoms_ptr(old_atoms)
        out = TrialEnergy()
        check(self.ctx.handle, lib().rg_intermolecular_energy_difference(self.handle, pn, len(n), po, len(o),
                                                                          ctypes.byref(out)),
              "rg_intermolecular_energy_difference")
        return out

    def update_molecules(self, first_atom: int, atoms):
        a, p = _atoms_ptr(atoms)
        check(self.ctx.handle, lib().rg_system_update_molecules(self.handle, first_atom, p, len(a)),
              "rg_system_update_molecules")

    def set_blocked_pockets(self, unit_cell, pockets):
        """pockets: (n, 4) centre as fractions of the framework unit cell and radius (Angstrom)."""
        pk = np.ascontiguousarray(pockets, dtype=np.float64).reshape(-1, 4)
        box = box_struct(unit_cell)
        check(self.ctx.handle, lib().rg_system_set_blocked_pockets(self.handle, ctypes.byref(box),
                                                                    ctypes.c_void_p(pk.ctypes.data), len(pk)),
              "rg_system_set_blocked_pockets")

    def set_external_field(self, surface_type: int, geometry=(5.0, 5.0, 0.0, 0.0), grid=None, grid_cell=None,
                           grid_dims=(0, 0, 0), grid_on_device: bool = False):
        """External field of the trial energies (rg_system_set_external_field); grid: host array or device pointer."""
        g = np.ascontiguousarray(geometry, dtype=np.float64).reshape(4)
        self._ext_geometry = g
        box = box_struct(grid_cell) if grid_cell is not None else None
        if grid is None:
            gptr = None
        elif grid_on_device:
            gptr = ctypes.c_void_p(int(grid))
        else:
            self._ext_grid = np.ascontiguousarray(grid, dtype=np.float64)
            gptr = ctypes.c_void_p(self._ext_grid.ctypes.data)
        check(self.ctx.handle, lib().rg_system_set_external_field(
            self.handle, surface_type, ctypes.c_void_p(g.ctypes.data), None if box is None else ctypes.byref(box),
            int(grid_dims[0]), int(grid_dims[1]), int(grid_dims[2]), gptr, 1 if grid_on_device else 0),
            "rg_system_set_external_field")


class EwaldBatch:
    """Structure factors of many systems sharing one Ewald state's k-vectors (rg_ewald_batch)."""

    def __init__(self, ewald: "Ewald", n_systems: int):
        self.ctx = ewald.ctx
        self.n = n_systems
        self.nk = ewald.n_kvectors
        h = ctypes.c_void_p()
        check(self.ctx.handle, lib().rg_ewald_batch_create(ewald.handle, n_systems, ctypes.byref(h)),
              "rg_ewald_batch_create")
        self.handle = h
        self.ctx.adopt(self)

    def close(self):
        if getattr(self, "handle", None):
            lib().rg_ewald_batch_destroy(self.handle)
            self.handle = None

    def set(self, system: int, sk=None):
        s = None if sk is None else np.ascontiguousarray(sk, dtype=np.float64)
        check(self.ctx.handle, lib().rg_ewald_batch_set(self.handle, system,
                                                        None if s is None else ctypes.c_void_p(s.ctypes.data)),
              "rg_ewald_batch_set")

    def get(self, system: int, which: int = 0) -> np.ndarray:
        out = np.empty(2 * self.nk)
        check(self.ctx.handle, lib().rg_ewald_batch_get(self.handle, system, which, ctypes.c_void_p(out.ctypes.data)),
              "rg_ewald_batch_get")
        return out

    def delta(self, atoms, max_atoms: int, n_new, n_old) -> np.ndarray:
        a, p = _atoms_ptr(atoms)
        nn = np.ascontiguousarray(n_new, dtype=np.int32)
        no = np.ascontiguousarray(n_old, dtype=np.int32)
        out = np.empty(self.n)
        check(self.ctx.handle, lib().rg_ewald_batch_delta(self.handle, p, max_atoms, ctypes.c_void_p(nn.ctypes.data),
                                                          ctypes.c_void_p(no.ctypes.data),
                                                          ctypes.c_void_p(out.ctypes.data)), "rg_ewald_batch_delta")
        return out

    def accept(self, mask):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        check(self.ctx.handle, lib().rg_ewald_batch_accept(self.handle, ctypes.c_void_p(m.ctypes.data)),
              "rg_ewald_batch_accept")

    def timing(self) -> tuple[float, float]:
        """Device time of the last delta in ms: (upload of the moved atoms, update kernel)."""
        up, k = ctypes.c_float(), ctypes.c_float()
        check(self.ctx.handle, lib().rg_ewald_batch_timing(self.handle, ctypes.byref(up), ctypes.byref(k)),
              "rg_ewald_batch_timing")
        return float(up.value), float(k.value)


class Gcmc:
    """Independent device-resident GCMC chains of one rigid component (rg_gcmc)."""

    def __init__(self, system: System, ewald, component, beta: float, fugacity: float, n_chains: int, seed: int = 1,
                 max_translation: float = 1.0, max_rotation: float = 0.5235987755982988,
                 probabilities=(1.0, 1.0, 1.0), n_first: int = 10, n_orient: int = 10, max_molecules: int = 256):
        self.ctx = system.ctx
        self.system = system
        self.ewald = ewald
        self.component = component
        self.n_chains = n_chains
        ff = system.ff
        c = GcmcComponent()
        c.n_atoms = component.n_atoms
        c.starting_bead = component.starting_bead
        types, charges = component.types(ff), component.charges(ff)
        for i in range(component.n_atoms):
            c.types[i] = int(types[i])
            c.charges[i] = float(charges[i])
            c.masses[i] = float(component.masses[i])
            for d in range(3):
                c.offsets[3 * i + d] = float(component.offsets[i][d])
        p = GcmcParams(beta, fugacity, ff.cutoff_framework_vdw, ff.cutoff_molecule_vdw, ff.cutoff_coulomb,
                       max_translation, max_rotation, probabilities[0], probabilities[1], probabilities[2], n_first,
                       n_orient, max_molecules, seed)
        h = ctypes.c_void_p()
        check(self.ctx.handle, lib().rg_gcmc_create(system.handle, ewald.handle if ewald is not None else None,
                                                    ctypes.byref(c), ctypes.byref(p), n_chains, ctypes.byref(h)),
              "rg_gcmc_create")
        self.handle = h
        self.ctx.adopt(self)
        self.max_molecules = max_molecules

    def close(self):
        if self.handle:
            lib().rg_gcmc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, moves: int, record: bool = True):
        check(self.ctx.handle, lib().rg_gcmc_run(self.handle, moves, 1 if record else 0), "rg_gcmc_run")

    def set_proposal(self, proposal, unit_cell=None):
        """Learned first-bead proposal (None: uniform positions)."""
        self._proposal = proposal
        if proposal is None:
            check(self.ctx.handle, lib().rg_gcmc_set_proposal(self.handle, None, None), "rg_gcmc_set_proposal")
        else:
            box = box_struct(unit_cell)
            check(self.ctx.handle, lib().rg_gcmc_set_proposal(self.handle, proposal.handle, ctypes.byref(box)),
                  "rg_gcmc_set_proposal")

    def results(self):
        out = (GcmcChainResult * self.n_chains)()
        check(self.ctx.handle, lib().rg_gcmc_results(self.handle, ctypes.cast(out, ctypes.c_void_p)),
              "rg_gcmc_results")
        return [out[i].as_dict() for i in range(self.n_chains)]

    def positions(self, chain: int) -> np.ndarray:
        cap = self.max_molecules * self.component.n_atoms
        buf = np.empty(3 * cap)
        n = ctypes.c_int32()
        check(self.ctx.handle, lib().rg_gcmc_get_positions(self.handle, chain, ctypes.c_void_p(buf.ctypes.data), cap,
                                                           ctypes.byref(n)), "rg_gcmc_get_positions")
        return buf[: 3 * n.value * self.component.n_atoms].reshape(-1, 3)


class Mlp:
    """The learned proposal's Fourier-feature MLP on the device (rg_mlp)."""

    def __init__(self, ctx: Context, seed: int = 1):
        self.ctx = ctx
        h = ctypes.c_void_p()
        check(ctx.handle, lib().rg_mlp_create(ctx.handle, seed, ctypes.byref(h)), "rg_mlp_create")
        self.handle = h
        ctx.adopt(self)
        self.n_params = lib().rg_mlp_num_params()

    def close(self):
        if self.handle:
            lib().rg_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        check(self.ctx.handle, lib().rg_mlp_get_params(self.handle, ctypes.c_void_p(out.ctypes.data), self.n_params),
              "rg_mlp_get_params")
        return out

    def set_params(self, theta):
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        check(self.ctx.handle, lib().rg_mlp_set_params(self.handle, ctypes.c_void_p(theta.ctypes.data), len(theta)),
              "rg_mlp_set_params")

    def loss_and_gradient(self, s_ptr: int, t_ptr: int, n: int):
        loss = ctypes.c_float()
        grad = np.empty(self.n_params, dtype=np.float32)
        check(self.ctx.handle, lib().rg_mlp_loss_and_gradient(self.handle, s_ptr, t_ptr, n, ctypes.byref(loss),
                                                              ctypes.c_void_p(grad.ctypes.data)),
              "rg_mlp_loss_and_gradient")
        return loss.value, grad

    def train(self, s_ptr: int, t_ptr: int, n: int, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 1):
        loss = ctypes.c_float()
        check(self.ctx.handle, lib().rg_mlp_train(self.handle, s_ptr, t_ptr, n, steps, batch, lr, seed,
                                                  ctypes.byref(loss)), "rg_mlp_train")
        return loss.value

    def evaluate(self, s_ptr: int, n: int, out_ptr: int):
        check(self.ctx.handle, lib().rg_mlp_evaluate(self.handle, s_ptr, n, out_ptr), "rg_mlp_evaluate")


def sample_targets(system: System, pseudo_atom: int, charge: float, beta: float, t_min: float, unit_cell, n: int,
                   seed: int, s_ptr: int, t_ptr: int):
    box = box_struct(unit_cell)
    check(system.ctx.handle, lib().rg_proposal_sample_targets(system.handle, pseudo_atom, charge, beta, t_min,
                                                              ctypes.byref(box), n, seed, s_ptr, t_ptr),
          "rg_proposal_sample_targets")


class Proposal:
    """A tabulated, exactly normalised first-bead proposal (rg_proposal) built from an Mlp."""

    def __init__(self, mlp: Mlp, cells_per_axis: int = 64, eps_uniform: float = 0.1):
        self.ctx = mlp.ctx
        h = ctypes.c_void_p()
        check(self.ctx.handle, lib().rg_proposal_create(mlp.handle, cells_per_axis, eps_uniform, ctypes.byref(h)),
              "rg_proposal_create")
        self.handle = h
        self.ctx.adopt(self)
        self.cells = cells_per_axis
        self.eps = eps_uniform

    def close(self):
        if self.handle:
            lib().rg_proposal_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def density(self, s) -> np.ndarray:
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(s))
        check(self.ctx.handle, lib().rg_proposal_density(self.handle, ctypes.c_void_p(s.ctypes.data), len(s),
                                                         ctypes.c_void_p(out.ctypes.data)), "rg_proposal_density")
        return out


class Alkane:
    """A batch of independent systems running GCMC of flexible chains (rg_alkane)."""

    def __init__(self, ctx: Context, ff: ForceField, systems, seed: int = 1):
        from .alkane import RgAlkaneChain, chain_struct

        class RgAlkaneSystem(ctypes.Structure):
            _fields_ = [("box", RgBox), ("framework", ctypes.c_void_p), ("n_framework", ctypes.c_int32),
                        ("max_molecules", ctypes.c_int32), ("chain", RgAlkaneChain), ("beta", ctypes.c_double),
                        ("fugacity", ctypes.c_double), ("w_ig", ctypes.c_double), ("max_translation", ctypes.c_double),
                        ("p_translation", ctypes.c_double), ("p_swap", ctypes.c_double)]

        self.ctx = ctx
        self.ff = ff
        self.systems = list(systems)
        n = len(self.systems)
        arr = (RgAlkaneSystem * n)()
        self._keep = []
        for i, q in enumerate(self.systems):
            fw = np.ascontiguousarray(q.framework, dtype=ATOM_DTYPE)
            self._keep.append(fw)
            arr[i].box = box_struct(q.cell)
            arr[i].framework = fw.ctypes.data if len(fw) else None
            arr[i].n_framework = len(fw)
            arr[i].max_molecules = q.max_molecules
            arr[i].chain = chain_struct(q.chain, ff)
            arr[i].beta, arr[i].fugacity, arr[i].w_ig = q.beta, q.fugacity, q.w_ig
            arr[i].max_translation, arr[i].p_translation, arr[i].p_swap = q.max_translation, q.p_translation, q.p_swap
        ffs = ff_struct(ff)
        h = ctypes.c_void_p()
        check(ctx.handle, lib().rg_alkane_create(ctx.handle, ctypes.byref(ffs), ctypes.cast(arr, ctypes.c_void_p), n,
                                                 seed, ctypes.byref(h)), "rg_alkane_create")
        self.handle = h
        ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().rg_alkane_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, moves_per_candidate: int = 8) -> dict:
        pl = AlkanePlan()
        check(self.ctx.handle, lib().rg_alkane_autotune(self.handle, moves_per_candidate, ctypes.byref(pl)),
              "rg_alkane_autotune")
        return pl.as_dict()

    def plan(self) -> dict:
        pl = AlkanePlan()
        check(self.ctx.handle, lib().rg_alkane_get_plan(self.handle, ctypes.byref(pl)), "rg_alkane_get_plan")
        return pl.as_dict()

    def set_plan(self, cluster_big=1, cluster_small=1, threads=128, split=0, moves_per_launch=64):
        pl = AlkanePlan(cluster_big, cluster_small, threads, split, moves_per_launch, 0, 0.0)
        check(self.ctx.handle, lib().rg_alkane_set_plan(self.handle, ctypes.byref(pl)), "rg_alkane_set_plan")

    def run(self, moves: int, record: bool = True):
        check(self.ctx.handle, lib().rg_alkane_run(self.handle, moves, 1 if record else 0), "rg_alkane_run")

    def launch_count(self) -> int:
        v = ctypes.c_int64()
        check(self.ctx.handle, lib().rg_alkane_launch_count(self.handle, ctypes.byref(v)), "rg_alkane_launch_count")
        return int(v.value)

    def pair_count(self) -> int:
        v = ctypes.c_uint64()
        check(self.ctx.handle, lib().rg_alkane_pair_count(self.handle, ctypes.byref(v)), "rg_alkane_pair_count")
        return int(v.value)

    def results(self):
        n = len(self.systems)
        out = (GcmcChainResult * n)()
        check(self.ctx.handle, lib().rg_alkane_results(self.handle, ctypes.cast(out, ctypes.c_void_p)),
              "rg_alkane_results")
        return [out[i].as_dict() for i in range(n)]

    def positions(self, system: int) -> np.ndarray:
        q = self.systems[system]
        cap = 3 * q.max_molecules * q.chain.n_beads
        buf = np.empty(cap)
        n = ctypes.c_int32()
        check(self.ctx.handle, lib().rg_alkane_get_positions(self.handle, system, ctypes.c_void_p(buf.ctypes.data),
                                                             cap, ctypes.byref(n)), "rg_alkane_get_positions")
        return buf[: 3 * n.value * q.chain.n_beads].reshape(n.value, q.chain.n_beads, 3)

    def set_positions(self, system: int, xyz, energy: float = 0.0):
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        nb = self.systems[system].chain.n_beads
        check(self.ctx.handle, lib().rg_alkane_set_positions(self.handle, system, ctypes.c_void_p(x.ctypes.data),
                                                             len(x) // (3 * nb), energy), "rg_alkane_set_positions")

    def bead_energies(self, system: int, xyz, types, skip: int = -1):
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        t = np.ascontiguousarray(types, dtype=np.int32)
        n = len(t)
        fw, mm, ov = np.empty(n), np.empty(n), np.empty(n, dtype=np.int32)
        check(self.ctx.handle, lib().rg_alkane_bead_energies(self.handle, system, ctypes.c_void_p(x.ctypes.data),
                                                             ctypes.c_void_p(t.ctypes.data), n, skip,
                                                             ctypes.c_void_p(fw.ctypes.data),
                                                             ctypes.c_void_p(mm.ctypes.data),
                                                             ctypes.c_void_p(ov.ctypes.data)),
              "rg_alkane_bead_energies")
        return fw, mm, ov


def alkane_grow_vacuum(ctx: Context, ff: ForceField, chain, beta: float, n: int, seed: int = 1, details: bool = False):
    """Chains grown in vacuum on the device: returns <W> (the ideal-gas Rosenbluth weight), or with details
    (<W>, w[n], theta[n, nb-2], cos_phi[n, nb-3])."""
    from .alkane import chain_struct

    c = chain_struct(chain, ff)
    ffs = ff_struct(ff)
    nb = chain.n_beads
    mean = ctypes.c_double()
    w = np.empty(n) if details else None
    th = np.empty(n * max(0, nb - 2)) if details else None
    cp = np.empty(n * max(0, nb - 3)) if details else None
    ptr = (lambda a: None if a is None or a.size == 0 else ctypes.c_void_p(a.ctypes.data))
    check(ctx.handle, lib().rg_alkane_grow_vacuum(ctx.handle, ctypes.byref(ffs), ctypes.byref(c), beta, n, seed,
                                                  ctypes.byref(mean), ptr(w), ptr(th), ptr(cp)),
          "rg_alkane_grow_vacuum")
    if not details:
        return mean.value
    return mean.value, w, th.reshape(n, max(0, nb - 2)), cp.reshape(n, max(0, nb - 3))


def component_struct(component, ff: ForceField) -> GcmcComponent:
    c = GcmcComponent()
    c.n_atoms = component.n_atoms
    c.starting_bead = component.starting_bead
    types, charges = component.types(ff), component.charges(ff)
    for i in range(component.n_atoms):
        c.types[i] = int(types[i])
        c.charges[i] = float(charges[i])
        c.masses[i] = float(component.masses[i])
        for d in range(3):
            c.offsets[3 * i + d] = float(component.offsets[i][d])
    return c


class Mixture:
    """One large system of several rigid components advanced on the whole GPU (rg_mixture)."""

    def __init__(self, system: System, ewald, components, beta: float, fugacities, xyz, comp, max_molecules: int,
                 seed: int = 1, probabilities=(1.0, 1.0, 1.0, 1.0), n_first: int = 10, n_orient: int = 10,
                 max_translation: float = 1.0, max_rotation: float = 0.5235987755982988, n_blocks: int = 0,
                 w_ig=None):
        self.ctx = system.ctx
        self.system = system
        self.components = list(components)
        ff = system.ff
        arr = (GcmcComponent * len(self.components))()
        for i, c in enumerate(self.components):
            arr[i] = component_struct(c, ff)
        p = MixtureParams()
        p.beta = beta
        for i, f in enumerate(fugacities):
            p.fugacity[i] = f
            p.w_ig[i] = 1.0 if w_ig is None else w_ig[i]
        p.cutoff_molecule_vdw, p.cutoff_coulomb = ff.cutoff_molecule_vdw, ff.cutoff_coulomb
        p.cutoff_framework_vdw = ff.cutoff_framework_vdw
        p.max_translation, p.max_rotation = max_translation, max_rotation
        p.p_translation, p.p_rotation, p.p_swap, p.p_identity = probabilities
        p.n_first_bead_trials, p.n_orientation_trials = n_first, n_orient
        p.max_molecules, p.n_blocks, p.seed = max_molecules, n_blocks, seed
        x = np.ascontiguousarray(xyz, dtype=np.float64)
        cc = np.ascontiguousarray(comp, dtype=np.int32)
        self.na = self.components[0].n_atoms
        self.max_molecules = max_molecules
        h = ctypes.c_void_p()
        check(self.ctx.handle, lib().rg_mixture_create(system.handle, ewald.handle if ewald is not None else None,
                                                       ctypes.cast(arr, ctypes.c_void_p), len(self.components),
                                                       ctypes.byref(p), ctypes.c_void_p(x.ctypes.data) if len(cc) else None,
                                                       ctypes.c_void_p(cc.ctypes.data) if len(cc) else None, len(cc),
                                                       ctypes.byref(h)), "rg_mixture_create")
        self.handle = h
        self.ctx.adopt(self)

    def close(self):
        if self.handle:
            lib().rg_mixture_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, energy: float, sk=None):
        s = None if sk is None else np.ascontiguousarray(sk, dtype=np.float64)
        check(self.ctx.handle, lib().rg_mixture_set_state(self.handle, energy,
                                                          None if s is None else ctypes.c_void_p(s.ctypes.data),
                                                          0 if s is None else len(s)), "rg_mixture_set_state")

    def run(self, moves: int, record: bool = True):
        check(self.ctx.handle, lib().rg_mixture_run(self.handle, moves, 1 if record else 0), "rg_mixture_run")

    def results(self) -> dict:
        r = MixtureResult()
        check(self.ctx.handle, lib().rg_mixture_results(self.handle, ctypes.byref(r)), "rg_mixture_results")
        return r.as_dict()

    @staticmethod
    def run_many(mixtures, moves: int, record: bool = True):
        """Several mixtures (one context, one CTA count) advanced by one cooperative launch (rg_mixture_run_many)."""
        arr = (ctypes.c_void_p * len(mixtures))(*[m.handle.value for m in mixtures])
        check(mixtures[0].ctx.handle, lib().rg_mixture_run_many(ctypes.cast(arr, ctypes.c_void_p), len(mixtures),
                                                                moves, 1 if record else 0), "rg_mixture_run_many")

    def set_wait_test(self, absent_cta: int, spin_limit: int):
        """Test of the bounded barrier wait (rg_mixture_set_wait_test): the next launch's waits give up by design."""
        check(self.ctx.handle, lib().rg_mixture_set_wait_test(self.handle, absent_cta, spin_limit),
              "rg_mixture_set_wait_test")

    def positions(self):
        xyz = np.empty(3 * self.max_molecules * self.na)
        comp = np.empty(self.max_molecules, dtype=np.int32)
        n = ctypes.c_int32()
        check(self.ctx.handle, lib().rg_mixture_get_positions(self.handle, ctypes.c_void_p(xyz.ctypes.data),
                                                              ctypes.c_void_p(comp.ctypes.data), self.max_molecules,
                                                              ctypes.byref(n)), "rg_mixture_get_positions")
        return xyz[: 3 * n.value * self.na].reshape(n.value, self.na, 3), comp[: n.value].copy()

    def structure_factors(self) -> np.ndarray:
        b, nk = ctypes.c_int32(), ctypes.c_int64()
        check(self.ctx.handle, lib().rg_mixture_info(self.handle, ctypes.byref(b), ctypes.byref(nk)), "rg_mixture_info")
        out = np.empty(2 * nk.value)
        check(self.ctx.handle, lib().rg_mixture_get_structure_factors(self.handle, ctypes.c_void_p(out.ctypes.data),
                                                                      len(out)), "rg_mixture_get_structure_factors")
        return out

    def info(self):
        b, nk = ctypes.c_int32(), ctypes.c_int64()
        check(self.ctx.handle, lib().rg_mixture_info(self.handle, ctypes.byref(b), ctypes.byref(nk)), "rg_mixture_info")
        return {"blocks": b.value, "n_kvectors": nk.value}

    def set_proposal(self, component: int, proposal, unit_cell=None):
        if proposal is None:
            check(self.ctx.handle, lib().rg_mixture_set_proposal(self.handle, component, None, None),
                  "rg_mixture_set_proposal")
        else:
            box = box_struct(unit_cell)
            check(self.ctx.handle, lib().rg_mixture_set_proposal(self.handle, component, proposal.handle,
                                                                 ctypes.byref(box)), "rg_mixture_set_proposal")

"""ctypes wrapper of the FP64 CPU oracle (oracle/_build/liboracle.so) — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu-baseline / reference arms import this module. It is the
checker the CUDA path is compared against; the product never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(quiet: bool = True) -> str:
    subprocess.run(["make", "-C", _HERE], check=True, capture_output=quiet)
    return _LIB_PATH


class OAtomPtr(ctypes.c_void_p):
    pass


class OBox(ctypes.Structure):
    _fields_ = [("cell", ctypes.c_double * 9), ("triclinic", ctypes.c_int32)]


class OFF(ctypes.Structure):
    _fields_ = [
        ("n_types", ctypes.c_int32),
        ("epsilon", ctypes.POINTER(ctypes.c_double)),
        ("sigma", ctypes.POINTER(ctypes.c_double)),
        ("shift", ctypes.POINTER(ctypes.c_double)),
        ("lj", ctypes.POINTER(ctypes.c_int32)),
        ("cutoff_framework_vdw", ctypes.c_double),
        ("cutoff_molecule_vdw", ctypes.c_double),
        ("cutoff_coulomb", ctypes.c_double),
        ("ewald_alpha", ctypes.c_double),
        ("kmax_x", ctypes.c_int32), ("kmax_y", ctypes.c_int32), ("kmax_z", ctypes.c_int32),
        ("recip_int_cutoff_sq", ctypes.c_uint64),
        ("recip_cutoff_sq", ctypes.c_double),
        ("overlap_criteria", ctypes.c_double),
        ("use_charge", ctypes.c_int32),
        ("omit_inter", ctypes.c_int32),
    ]


ENERGY_FIELDS = ["framework_molecule_vdw", "framework_molecule_charge", "molecule_molecule_vdw",
                 "molecule_molecule_charge", "ewald_fourier", "ewald_self", "ewald_exclusion"]


class OEnergy(ctypes.Structure):
    _fields_ = [(f, ctypes.c_double) for f in ENERGY_FIELDS] + [
        ("dudlambda_vdw", ctypes.c_double * 4), ("dudlambda_charge", ctypes.c_double * 4),
        ("dudlambda_ewald", ctypes.c_double * 4)]

    def as_dict(self):
        d = {f: getattr(self, f) for f in ENERGY_FIELDS}
        d["dudlambda_vdw"] = list(self.dudlambda_vdw)
        d["dudlambda_charge"] = list(self.dudlambda_charge)
        d["dudlambda_ewald"] = list(self.dudlambda_ewald)
        return d


def use_release_build(quiet: bool = True) -> str:
    """Switches this module to the oracle built with the reference's release flags (-O3 -ffast-math, plus
    -march=native), compiled on this machine: the timed CPU baseline. The strict build stays the parity oracle of the
    tests; call this only from a process that times the baseline."""
    global _lib, _LIB_PATH
    import hashlib

    cpu = ""
    if os.path.exists("/proc/cpuinfo"):
        for line in open("/proc/cpuinfo"):
            if line.startswith(("model name", "flags")):
                cpu += line
            if cpu.count("\n") >= 2:
                break
    tag = hashlib.sha1(cpu.encode()).hexdigest()[:12]
    rel = os.path.join("_build", "release_" + tag)
    subprocess.run(["make", "-C", _HERE, "-j4", "release", f"RELEASE_DIR={rel}"], check=True, capture_output=quiet)
    _LIB_PATH = os.path.join(_HERE, rel, "liboracle_release.so")
    _lib = None
    lib()
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d, i32, i64, vp = ctypes.c_double, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p
        L.oracle_energy_to_kelvin.restype = d
        L.oracle_kelvin_to_energy.restype = d
        L.oracle_coulomb_factor.restype = d
        L.oracle_make_tricubic_grid.argtypes = [i32, P(OFF), P(OBox), vp, i32, i32, d, i32, i32, i32, vp, i64, i32, vp]
        L.oracle_make_tricubic_grid.restype = i32
        L.oracle_grid_pair_count.argtypes = [i32, P(OFF), P(OBox), vp, i32, i32, d, i32, i32, i32, vp, i64, i32]
        L.oracle_grid_pair_count.restype = i64
        L.oracle_tricubic_fractional_at_position.argtypes = [i32, P(OFF), P(OBox), vp, i32, P(OBox), vp, i32, vp]
        L.oracle_tricubic_matrix.argtypes = [vp]
        L.oracle_triquintic_fractional_at_position.argtypes = [i32, P(OFF), P(OBox), vp, i32, P(OBox), vp, i32, i32,
                                                               vp]
        L.oracle_make_triquintic_grid.argtypes = [i32, P(OFF), P(OBox), vp, i32, i32, d, i32, i32, i32, i32, vp, i64,
                                                  i32, vp]
        L.oracle_make_triquintic_grid.restype = i32
        L.oracle_triquintic_interpolate.argtypes = [vp, i32, i32, i32, P(OBox), vp, vp]
        L.oracle_triquintic_interpolate.restype = d
        L.oracle_interpolant_from_corners.argtypes = [i32, vp, vp, vp]
        L.oracle_interpolant_from_corners.restype = d
        L.oracle_triquintic_matrix.argtypes = [vp]
        L.oracle_grid_validate_triquintic.argtypes = [P(OFF), P(OBox), vp, i32, P(OBox), i32, i32, i32, i32, vp, vp, d, d,
                                                      vp, i64, vp]
        L.oracle_grid_interpolate.argtypes = [vp, i32, i32, i32, P(OBox), vp]
        L.oracle_grid_interpolate.restype = d
        L.oracle_grid_validate.argtypes = [P(OFF), P(OBox), vp, i32, P(OBox), i32, i32, i32, i32, vp, vp, d, d, vp,
                                           ctypes.c_int64, vp]
        L.oracle_pair_vdw.argtypes = [P(OFF), d, d, d, i32, i32, vp]
        L.oracle_pair_coulomb.argtypes = [P(OFF), d, d, d, d, d, vp]
        L.oracle_cbmc_framework_molecule.argtypes = [P(OFF), P(OBox), vp, i32, i32, i32, P(OBox), vp, i32, d, d, vp,
                                                     i32, i32, P(OEnergy)]
        L.oracle_cbmc_framework_molecule.restype = i32
        L.oracle_cbmc_intermolecular.argtypes = [P(OFF), P(OBox), vp, i32, d, d, vp, i32, i32, i64, P(OEnergy)]
        L.oracle_cbmc_intermolecular.restype = i32
        L.oracle_framework_molecule_energy_difference.argtypes = [P(OFF), P(OBox), vp, i32, i32, i32, P(OBox), vp, i32,
                                                                  i32, vp, i32, vp, i32, P(OEnergy)]
        L.oracle_framework_molecule_energy_difference.restype = i32
        L.oracle_intermolecular_energy_difference.argtypes = [P(OFF), P(OBox), vp, i32, vp, i32, vp, i32, P(OEnergy)]
        L.oracle_intermolecular_energy_difference.restype = i32
        L.oracle_inside_blocked_pockets.argtypes = [P(OBox), vp, i32, vp, i32]
        L.oracle_inside_blocked_pockets.restype = i32
        L.oracle_external_field_energy.argtypes = [i32, vp, P(OBox), vp, i32, i32, i32, P(OBox), vp, i32, i32,
                                                   P(ctypes.c_double)]
        L.oracle_external_field_energy.restype = i32
        L.oracle_ewald_kvectors.argtypes = [P(OFF), P(OBox), vp, vp, vp]
        L.oracle_ewald_kvectors.restype = i64
        L.oracle_ewald_rigid.argtypes = [P(OFF), P(OBox), vp, i32, vp]
        L.oracle_ewald_fourier_energy.argtypes = [P(OFF), P(OBox), vp, vp, i32, vp, i32, d, vp, P(OEnergy)]
        L.oracle_ewald_delta.argtypes = [P(OFF), P(OBox), vp, vp, i32, vp, i32, d, vp, vp, P(OEnergy)]
        L.oracle_ewald_delta_parallel.argtypes = [P(OFF), P(OBox), vp, vp, i64, vp, vp, i32, vp, i32, vp, i32]
        L.oracle_ewald_delta_parallel.restype = d
        L.oracle_ewald_single_ion.argtypes = [P(OFF), P(OBox), vp, d]
        L.oracle_ewald_single_ion.restype = d
        L.oracle_select_trial.argtypes = [vp, i32, d]
        L.oracle_select_trial.restype = i32
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def off(ff) -> OFF:
    """OFF struct from a raspa3_b200.forcefield.ForceField (keeps the arrays alive on the struct)."""
    eps = np.ascontiguousarray(ff.epsilon, dtype=np.float64)
    sig = np.ascontiguousarray(ff.sigma, dtype=np.float64)
    sh = np.ascontiguousarray(ff.shift, dtype=np.float64)
    lj = np.ascontiguousarray(ff.lj, dtype=np.int32)
    P = ctypes.POINTER
    s = OFF(ff.n_types, eps.ctypes.data_as(P(ctypes.c_double)), sig.ctypes.data_as(P(ctypes.c_double)),
            sh.ctypes.data_as(P(ctypes.c_double)), lj.ctypes.data_as(P(ctypes.c_int32)),
            ff.cutoff_framework_vdw, ff.cutoff_molecule_vdw, ff.cutoff_coulomb, ff.ewald_alpha,
            int(ff.kmax[0]), int(ff.kmax[1]), int(ff.kmax[2]), int(ff.recip_int_cutoff_sq), ff.recip_cutoff_sq,
            ff.overlap_criteria, 1 if ff.use_charge else 0, 1 if ff.omit_inter else 0)
    s._keep = (eps, sig, sh, lj)
    return s


def obox(cell, triclinic=None) -> OBox:
    cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
    if triclinic is None:
        triclinic = bool(np.any(cell - np.diag(np.diag(cell)) != 0.0))
    b = OBox()
    for i in range(9):
        b.cell[i] = float(cell.reshape(-1)[i])
    b.triclinic = 1 if triclinic else 0
    return b


def energy_to_kelvin() -> float:
    return lib().oracle_energy_to_kelvin()


def make_grid(grid_type, ff, cell, atoms, probe_type, cutoff, dims, points=None, threads=0):
    """Full tricubic grid (flat, reference layout) or the 8 values at the listed flat point indices."""
    nx, ny, nz = dims
    o, b = off(ff), obox(cell)
    atoms = np.ascontiguousarray(atoms)
    if points is None:
        out = np.empty(8 * nx * ny * nz)
        lib().oracle_make_tricubic_grid(grid_type, o, b, _ptr(atoms), len(atoms), probe_type, cutoff, nx, ny, nz,
                                        None, 0, threads, _ptr(out))
        return out
    pts = np.ascontiguousarray(points, dtype=np.int64)
    out = np.empty((len(pts), 8))
    lib().oracle_make_tricubic_grid(grid_type, o, b, _ptr(atoms), len(atoms), probe_type, cutoff, nx, ny, nz,
                                    _ptr(pts), len(pts), threads, _ptr(out))
    return out


def grid_pair_count(grid_type, ff, cell, atoms, probe_type, cutoff, dims, points=None, threads=0) -> int:
    nx, ny, nz = dims
    atoms = np.ascontiguousarray(atoms)
    if points is None:
        return lib().oracle_grid_pair_count(grid_type, off(ff), obox(cell), _ptr(atoms), len(atoms), probe_type,
                                            cutoff, nx, ny, nz, None, 0, threads)
    pts = np.ascontiguousarray(points, dtype=np.int64)
    return lib().oracle_grid_pair_count(grid_type, off(ff), obox(cell), _ptr(atoms), len(atoms), probe_type, cutoff,
                                        nx, ny, nz, _ptr(pts), len(pts), threads)


def tricubic_fractional(grid_type, ff, super_cell, pos, type_a, unit_cell, super_atoms):
    out = np.empty(8)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    sa = np.ascontiguousarray(super_atoms)
    lib().oracle_tricubic_fractional_at_position(grid_type, off(ff), obox(super_cell), _ptr(p), type_a,
                                                 obox(unit_cell), _ptr(sa), len(sa), _ptr(out))
    return out


def tricubic_matrix() -> np.ndarray:
    m = np.empty(64 * 64)
    lib().oracle_tricubic_matrix(_ptr(m))
    return m.reshape(64, 64)


def make_grid_triquintic(grid_type, ff, cell, atoms, probe_type, cutoff, dims, points=None, threads=0,
                         reference_rectangular=False):
    """Triquintic grid (27 values per point, flat reference layout) or the 27 values at the listed flat indices."""
    nx, ny, nz = dims
    o, b = off(ff), obox(cell)
    atoms = np.ascontiguousarray(atoms)
    rr = 1 if reference_rectangular else 0
    if points is None:
        out = np.empty(27 * nx * ny * nz)
        lib().oracle_make_triquintic_grid(grid_type, o, b, _ptr(atoms), len(atoms), probe_type, cutoff, nx, ny, nz, rr,
                                          None, 0, threads, _ptr(out))
        return out
    pts = np.ascontiguousarray(points, dtype=np.int64)
    out = np.empty((len(pts), 27))
    lib().oracle_make_triquintic_grid(grid_type, o, b, _ptr(atoms), len(atoms), probe_type, cutoff, nx, ny, nz, rr,
                                      _ptr(pts), len(pts), threads, _ptr(out))
    return out


def triquintic_fractional(grid_type, ff, super_cell, pos, type_a, unit_cell, super_atoms, reference_rectangular=False,
                          triclinic=None):
    out = np.empty(27)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    sa = np.ascontiguousarray(super_atoms)
    lib().oracle_triquintic_fractional_at_position(grid_type, off(ff), obox(super_cell, triclinic), _ptr(p), type_a,
                                                   obox(unit_cell, triclinic), _ptr(sa), len(sa),
                                                   1 if reference_rectangular else 0, _ptr(out))
    return out


def interpolate_triquintic(grid, dims, cell, pos):
    """(value, Cartesian gradient) of a triquintic grid at pos."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    grad = np.empty(3)
    v = lib().oracle_triquintic_interpolate(_ptr(g), dims[0], dims[1], dims[2], obox(cell), _ptr(p), _ptr(grad))
    return v, grad


def interpolant_from_corners(scheme, X, s):
    """(value, d/ds) of one cell's interpolating polynomial from its corner data (scheme 8 or 27)."""
    x = np.ascontiguousarray(X, dtype=np.float64)
    sv = np.ascontiguousarray(s, dtype=np.float64)
    ds = np.empty(3)
    v = lib().oracle_interpolant_from_corners(scheme, _ptr(x), _ptr(sv), _ptr(ds))
    return v, ds


def triquintic_matrix() -> np.ndarray:
    m = np.empty(216 * 216)
    lib().oracle_triquintic_matrix(_ptr(m))
    return m.reshape(216, 216)


def grid_validate(ff, unit_cell, unit_atoms, simulation_cell, probe_type, dims, vdw_grid, ewald_grid, probe_charge,
                  weight_beta, points):
    """The grid test of System::createFrameworkInterpolationGrids (tricubic) at the given points (n x 3 fractions of
    the simulation box): 36 values, the Boltzmann-weighted sums of the VDW (0..16) and charge (17..33) terms and the
    two point counts."""
    nx, ny, nz = dims
    atoms = np.ascontiguousarray(unit_atoms)
    pts = np.ascontiguousarray(points, dtype=np.float64)
    vg = np.ascontiguousarray(vdw_grid, dtype=np.float64)
    eg = None if ewald_grid is None else np.ascontiguousarray(ewald_grid, dtype=np.float64)
    out = np.zeros(36)
    lib().oracle_grid_validate(off(ff), obox(unit_cell), _ptr(atoms), len(atoms), obox(simulation_cell), probe_type,
                               nx, ny, nz, _ptr(vg), _ptr(eg), probe_charge, weight_beta, _ptr(pts), len(pts),
                               _ptr(out))
    return out


def grid_validate_triquintic(ff, unit_cell, unit_atoms, simulation_cell, probe_type, dims, vdw_grid, ewald_grid,
                             probe_charge, weight_beta, points):
    """The grid test of the triquintic scheme at the given points: 84 values (the 36 of grid_validate, then 24 VDW and
    24 charge Hessian sums)."""
    nx, ny, nz = dims
    atoms = np.ascontiguousarray(unit_atoms)
    pts = np.ascontiguousarray(points, dtype=np.float64)
    vg = np.ascontiguousarray(vdw_grid, dtype=np.float64)
    eg = None if ewald_grid is None else np.ascontiguousarray(ewald_grid, dtype=np.float64)
    out = np.zeros(84)
    lib().oracle_grid_validate_triquintic(off(ff), obox(unit_cell), _ptr(atoms), len(atoms), obox(simulation_cell),
                                          probe_type, nx, ny, nz, _ptr(vg), _ptr(eg), probe_charge, weight_beta,
                                          _ptr(pts), len(pts), _ptr(out))
    return out


def interpolate(grid, dims, cell, pos) -> float:
    g = np.ascontiguousarray(grid, dtype=np.float64)
    p = np.ascontiguousarray(pos, dtype=np.float64)
    return lib().oracle_grid_interpolate(_ptr(g), dims[0], dims[1], dims[2], obox(cell), _ptr(p))


def cbmc_framework_molecule(ff, cell, fw_atoms, atoms, cutoff_vdw, cutoff_coulomb, grids=None, grid_dims=None,
                            grid_cell=None, skip=-1):
    """Returns (ok, energy dict). grids: list of length n_types+1 of flat grids or None."""
    e = OEnergy()
    fw = np.ascontiguousarray(fw_atoms)
    at = np.ascontiguousarray(atoms)
    gptr = None
    keep = None
    gnx = gny = gnz = 0
    gbox = None
    if grids is not None:
        arr = (ctypes.c_void_p * len(grids))()
        keep = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in grids]
        for i, g in enumerate(keep):
            arr[i] = None if g is None else g.ctypes.data
        gptr = ctypes.cast(arr, ctypes.c_void_p)
        gnx, gny, gnz = grid_dims
        gbox = obox(grid_cell if grid_cell is not None else cell)
    ok = lib().oracle_cbmc_framework_molecule(off(ff), obox(cell), gptr, gnx, gny, gnz, gbox, _ptr(fw), len(fw),
                                              cutoff_vdw, cutoff_coulomb, _ptr(at), len(at), skip, ctypes.byref(e))
    del keep
    return bool(ok), e.as_dict()


def cbmc_intermolecular(ff, cell, molecule_atoms, atoms, cutoff_vdw, cutoff_coulomb, skip=-1, skip_background=-1):
    e = OEnergy()
    ma = np.ascontiguousarray(molecule_atoms)
    at = np.ascontiguousarray(atoms)
    ok = lib().oracle_cbmc_intermolecular(off(ff), obox(cell), _ptr(ma), len(ma), cutoff_vdw, cutoff_coulomb,
                                          _ptr(at), len(at), skip, skip_background, ctypes.byref(e))
    return bool(ok), e.as_dict()


def _grid_table(grids):
    """(pointer to an array of grid pointers, arrays kept alive) for a list of flat grids or None entries."""
    if grids is None:
        return None, None
    arr = (ctypes.c_void_p * len(grids))()
    keep = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in grids]
    for i, g in enumerate(keep):
        arr[i] = None if g is None else g.ctypes.data
    return ctypes.cast(arr, ctypes.c_void_p), (arr, keep)


def framework_molecule_energy_difference(ff, cell, fw_atoms, new_atoms, old_atoms, grids=None, grid_dims=None,
                                         grid_cell=None, charge_method_ewald=True):
    """Interactions::computeFrameworkMoleculeEnergyDifference: (ok, energy dict of E(new) - E(old))."""
    e = OEnergy()
    fw, na, oa = (np.ascontiguousarray(x) for x in (fw_atoms, new_atoms, old_atoms))
    gptr, keep = _grid_table(grids)
    gnx, gny, gnz = grid_dims if grid_dims is not None else (0, 0, 0)
    gbox = obox(grid_cell if grid_cell is not None else cell) if grids is not None else None
    ok = lib().oracle_framework_molecule_energy_difference(off(ff), obox(cell), gptr, gnx, gny, gnz, gbox, _ptr(fw),
                                                           len(fw), 1 if charge_method_ewald else 0, _ptr(na), len(na),
                                                           _ptr(oa), len(oa), ctypes.byref(e))
    del keep
    return bool(ok), e.as_dict()


def intermolecular_energy_difference(ff, cell, molecule_atoms, new_atoms, old_atoms):
    """Interactions::computeInterMolecularEnergyDifference: (ok, energy dict of E(new) - E(old))."""
    e = OEnergy()
    ma, na, oa = (np.ascontiguousarray(x) for x in (molecule_atoms, new_atoms, old_atoms))
    ok = lib().oracle_intermolecular_energy_difference(off(ff), obox(cell), _ptr(ma), len(ma), _ptr(na), len(na),
                                                       _ptr(oa), len(oa), ctypes.byref(e))
    return bool(ok), e.as_dict()


def inside_blocked_pockets(unit_cell, pockets, atoms) -> bool:
    """CBMC::insideBlockedPockets; pockets: (n, 4) fractional centre and radius."""
    pk = np.ascontiguousarray(pockets, dtype=np.float64).reshape(-1, 4)
    at = np.ascontiguousarray(atoms)
    return bool(lib().oracle_inside_blocked_pockets(obox(unit_cell), _ptr(pk), len(pk), _ptr(at), len(at)))


def external_field_energy(surface_type, geometry, cell, atoms, grid=None, grid_dims=None, grid_cell=None, skip=-1):
    """CBMC::computeExternalFieldEnergy: (ok, energy); ok False where a confinement surface returns nullopt."""
    g = np.asarray(geometry, dtype=np.float64).reshape(4)
    at = np.ascontiguousarray(atoms)
    gd = None if grid is None else np.ascontiguousarray(grid, dtype=np.float64)
    gnx, gny, gnz = grid_dims if grid_dims is not None else (0, 0, 0)
    e = ctypes.c_double()
    ok = lib().oracle_external_field_energy(int(surface_type), _ptr(g), obox(cell), _ptr(gd), gnx, gny, gnz,
                                            obox(grid_cell if grid_cell is not None else cell), _ptr(at), len(at),
                                            skip, ctypes.byref(e))
    return bool(ok), e.value


def pair_vdw(ff, sa, sb, rr, ta, tb):
    out = np.empty(2)
    lib().oracle_pair_vdw(off(ff), sa, sb, rr, ta, tb, _ptr(out))
    return out


def pair_coulomb(ff, sa, sb, r, qa, qb):
    out = np.empty(2)
    lib().oracle_pair_coulomb(off(ff), sa, sb, r, qa, qb, _ptr(out))
    return out


def ewald_kvectors(ff, cell):
    o, b = off(ff), obox(cell)
    n = lib().oracle_ewald_kvectors(o, b, None, None, None)
    kv = np.empty((n, 3), dtype=np.int32)
    temp = np.empty(n)
    s = ctypes.c_double()
    lib().oracle_ewald_kvectors(o, b, _ptr(kv), _ptr(temp), ctypes.c_void_p(ctypes.addressof(s)))
    return kv, temp, s.value


def ewald_rigid(ff, cell, fw_atoms):
    n = ewald_kvectors(ff, cell)[0].shape[0]
    out = np.zeros(2 * n)
    fw = np.ascontiguousarray(fw_atoms)
    lib().oracle_ewald_rigid(off(ff), obox(cell), _ptr(fw), len(fw), _ptr(out))
    return out


def ewald_fourier_energy(ff, cell, atoms, molecule_sizes, s_rigid=None, net_charge_framework=0.0):
    n = ewald_kvectors(ff, cell)[0].shape[0]
    stored = np.zeros(10 * n)
    at = np.ascontiguousarray(atoms)
    ms = np.ascontiguousarray(molecule_sizes, dtype=np.int32)
    e = OEnergy()
    sr = None if s_rigid is None else np.ascontiguousarray(s_rigid, dtype=np.float64)
    lib().oracle_ewald_fourier_energy(off(ff), obox(cell), _ptr(sr), _ptr(at), len(at), _ptr(ms), len(ms),
                                      net_charge_framework, _ptr(stored), ctypes.byref(e))
    return e.as_dict(), stored


def ewald_delta(ff, cell, stored, new_atoms, old_atoms, net_charge=0.0, net_charge_derivative_ext=None):
    trial = np.zeros_like(stored)
    na = np.ascontiguousarray(new_atoms)
    oa = np.ascontiguousarray(old_atoms)
    e = OEnergy()
    nd = None if net_charge_derivative_ext is None else np.ascontiguousarray(net_charge_derivative_ext, np.float64)
    st = np.ascontiguousarray(stored, dtype=np.float64)
    lib().oracle_ewald_delta(off(ff), obox(cell), _ptr(st), _ptr(na), len(na), _ptr(oa), len(oa), net_charge,
                             _ptr(nd), _ptr(trial), ctypes.byref(e))
    return e.as_dict(), trial


class EwaldDeltaParallel:
    """The k loop of energyDifferenceEwaldFourier on all host cores (OpenMP over a precomputed k table): the
    "restated reference loop, parallelised by us" CPU baseline of one Fourier difference."""

    def __init__(self, ff, cell, threads=0):
        self.off, self.box = off(ff), obox(cell)
        self.kvec, self.temp, _ = ewald_kvectors(ff, cell)
        self.threads = threads

    def __call__(self, stored, new_atoms, old_atoms, trial=None):
        st = np.ascontiguousarray(stored, dtype=np.float64)
        na, oa = np.ascontiguousarray(new_atoms), np.ascontiguousarray(old_atoms)
        return lib().oracle_ewald_delta_parallel(self.off, self.box, _ptr(self.kvec), _ptr(self.temp), len(self.temp),
                                                 _ptr(st), _ptr(na), len(na), _ptr(oa), len(oa), _ptr(trial),
                                                 self.threads)


def ewald_single_ion(ff, cell, pos, charge) -> float:
    p = np.ascontiguousarray(pos, dtype=np.float64)
    return lib().oracle_ewald_single_ion(off(ff), obox(cell), _ptr(p), charge)


def select_trial(log_boltzmann, uniform) -> int:
    lb = np.ascontiguousarray(log_boltzmann, dtype=np.float64)
    return lib().oracle_select_trial(_ptr(lb), len(lb), uniform)


class OGcmcSetup(ctypes.Structure):
    _fields_ = [
        ("ff", ctypes.POINTER(OFF)),
        ("box", OBox),
        ("grid_cell", OBox),
        ("gnx", ctypes.c_int32), ("gny", ctypes.c_int32), ("gnz", ctypes.c_int32),
        ("grids", ctypes.c_void_p),
        ("s_framework", ctypes.c_void_p),
        ("n_atoms", ctypes.c_int32),
        ("starting_bead", ctypes.c_int32),
        ("offsets", ctypes.c_double * 24),
        ("masses", ctypes.c_double * 8),
        ("types", ctypes.c_int32 * 8),
        ("charges", ctypes.c_double * 8),
        ("beta", ctypes.c_double),
        ("fugacity", ctypes.c_double),
        ("max_translation", ctypes.c_double),
        ("max_rotation", ctypes.c_double),
        ("p_translation", ctypes.c_double),
        ("p_rotation", ctypes.c_double),
        ("p_swap", ctypes.c_double),
        ("n_first_bead_trials", ctypes.c_int32),
        ("n_orientation_trials", ctypes.c_int32),
        ("max_molecules", ctypes.c_int32),
        ("use_ewald", ctypes.c_int32),
    ]


class OGcmcResult(ctypes.Structure):
    _fields_ = [
        ("n_molecules", ctypes.c_int64),
        ("running_energy", ctypes.c_double),
        ("recomputed_energy", ctypes.c_double),
        ("sum_n", ctypes.c_double),
        ("sum_n2", ctypes.c_double),
        ("sum_energy", ctypes.c_double),
        ("samples", ctypes.c_int64),
        ("attempted", ctypes.c_int64 * 4),
        ("accepted", ctypes.c_int64 * 4),
        ("block_n", ctypes.c_double * 5),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f not in ("attempted", "accepted", "block_n")}
        d["attempted"] = list(self.attempted)
        d["accepted"] = list(self.accepted)
        d["block_n"] = list(self.block_n)
        return d


def gcmc_run(ff, cell, component, beta, fugacity, n_chains, steps, equilibration=0, seed=1, threads=0, grids=None,
             grid_dims=None, grid_cell=None, s_framework=None, use_ewald=True, max_translation=1.0,
             max_rotation=0.5235987755982988, probabilities=(1.0, 1.0, 1.0), n_first=10, n_orient=10,
             max_molecules=512):
    """Independent GCMC chains of one rigid component; returns (list of result dicts, seconds)."""
    L = lib()
    if not hasattr(L, "_gcmc_declared"):
        L.oracle_gcmc_run.argtypes = [ctypes.POINTER(OGcmcSetup), ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L._gcmc_declared = True
    o = off(ff)
    s = OGcmcSetup()
    s.ff = ctypes.pointer(o)
    s.box = obox(cell)
    keep = [o]
    if grids is not None:
        arr = (ctypes.c_void_p * len(grids))()
        gk = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in grids]
        for i, g in enumerate(gk):
            arr[i] = None if g is None else g.ctypes.data
        keep += [arr, gk]
        s.grids = ctypes.cast(arr, ctypes.c_void_p)
        s.gnx, s.gny, s.gnz = grid_dims
        s.grid_cell = obox(grid_cell)
    if s_framework is not None:
        sf = np.ascontiguousarray(s_framework, dtype=np.float64)
        keep.append(sf)
        s.s_framework = sf.ctypes.data
    n = component.n_atoms
    s.n_atoms = n
    s.starting_bead = component.starting_bead
    types = component.types(ff)
    charges = component.charges(ff)
    for i in range(n):
        for d in range(3):
            s.offsets[3 * i + d] = float(component.offsets[i][d])
        s.masses[i] = float(component.masses[i])
        s.types[i] = int(types[i])
        s.charges[i] = float(charges[i])
    s.beta = beta
    s.fugacity = fugacity
    s.max_translation = max_translation
    s.max_rotation = max_rotation
    s.p_translation, s.p_rotation, s.p_swap = probabilities
    s.n_first_bead_trials = n_first
    s.n_orientation_trials = n_orient
    s.max_molecules = max_molecules
    s.use_ewald = 1 if use_ewald else 0
    out = (OGcmcResult * n_chains)()
    secs = ctypes.c_double()
    L.oracle_gcmc_run(ctypes.byref(s), n_chains, steps, equilibration, seed, threads, ctypes.cast(out, ctypes.c_void_p),
                      ctypes.c_void_p(ctypes.addressof(secs)))
    del keep
    return [out[i].as_dict() for i in range(n_chains)], secs.value


# ---- flexible alkane GCMC (oracle/alkane.cpp) ----
class OAlkane(ctypes.Structure):
    _fields_ = [("n_beads", ctypes.c_int32), ("types", ctypes.c_int32 * 8), ("bond_length", ctypes.c_double),
                ("bend_k", ctypes.c_double), ("bend_theta0", ctypes.c_double), ("torsion", ctypes.c_double * 4),
                ("n_first_bead_trials", ctypes.c_int32), ("n_trial_directions", ctypes.c_int32),
                ("n_torsion_trials", ctypes.c_int32), ("n_moves_per_open_bead", ctypes.c_int32)]


class OAlkaneSetup(ctypes.Structure):
    _fields_ = [("ff", ctypes.POINTER(OFF)), ("box", OBox), ("framework", ctypes.c_void_p),
                ("n_framework", ctypes.c_int32), ("chain", OAlkane), ("beta", ctypes.c_double),
                ("fugacity", ctypes.c_double), ("w_ig", ctypes.c_double), ("max_translation", ctypes.c_double),
                ("p_translation", ctypes.c_double), ("p_swap", ctypes.c_double), ("max_molecules", ctypes.c_int32)]


def _alkane_lib():
    L = lib()
    if not hasattr(L, "_alkane_declared"):
        P, vp, i32, i64, d = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.oracle_alkane_run.argtypes = [vp, i32, i64, i64, ctypes.c_uint64, i32, vp, vp, vp, vp, vp]
        L.oracle_alkane_grow_vacuum.argtypes = [P(OFF), P(OAlkane), d, i64, ctypes.c_uint64, i32, vp, vp, vp]
        L.oracle_alkane_energy.argtypes = [P(OAlkaneSetup), vp, i32, vp]
        L.oracle_alkane_bead_energies.argtypes = [P(OAlkaneSetup), vp, i32, vp, vp, i32, i32, vp, vp, vp]
        L._alkane_declared = True
    return L


def oalkane(chain, ff) -> OAlkane:
    """OAlkane from a raspa3_b200.alkane.AlkaneChain (internal units)."""
    from raspa3_b200.alkane import chain_struct

    c = chain_struct(chain, ff)
    o = OAlkane()
    o.n_beads = c.n_beads
    for i in range(8):
        o.types[i] = c.types[i]
    o.bond_length, o.bend_k, o.bend_theta0 = c.bond_length, c.bend_k, c.bend_theta0
    for k in range(4):
        o.torsion[k] = c.torsion[k]
    o.n_first_bead_trials, o.n_trial_directions = c.n_first_bead_trials, c.n_trial_directions
    o.n_torsion_trials = c.n_torsion_trials
    o.n_moves_per_open_bead = chain.n_moves_per_open_bead
    return o


def _alkane_setups(ff, systems):
    o = off(ff)
    arr = (OAlkaneSetup * len(systems))()
    keep = [o]
    for i, q in enumerate(systems):
        fw = np.ascontiguousarray(q.framework)
        keep.append(fw)
        arr[i].ff = ctypes.pointer(o)
        arr[i].box = obox(q.cell)
        arr[i].framework = fw.ctypes.data if len(fw) else None
        arr[i].n_framework = len(fw)
        arr[i].chain = oalkane(q.chain, ff)
        arr[i].beta, arr[i].fugacity, arr[i].w_ig = q.beta, q.fugacity, q.w_ig
        arr[i].max_translation, arr[i].p_translation, arr[i].p_swap = q.max_translation, q.p_translation, q.p_swap
        arr[i].max_molecules = q.max_molecules
    return arr, keep


def alkane_run(ff, systems, steps, equilibration=0, seed=1, threads=0, initial=None):
    """One oracle GCMC chain per system; returns (result dicts, final positions per system, seconds).
    initial: optional list of starting positions per system (arrays [n, nb, 3])."""
    L = _alkane_lib()
    arr, keep = _alkane_setups(ff, systems)
    n = len(systems)
    out = (OGcmcResult * n)()
    offs = []
    o = 0
    for q in systems:
        offs.append(o)
        o += q.max_molecules * q.chain.n_beads * 3
    xyz = np.zeros(o)
    xin, nin = None, None
    if initial is not None:
        xin = np.zeros(o)
        nin = np.zeros(n, dtype=np.int32)
        for i, x in enumerate(initial):
            x = np.asarray(x, dtype=np.float64).reshape(-1)
            xin[offs[i]: offs[i] + len(x)] = x
            nin[i] = len(x) // (3 * systems[i].chain.n_beads)
    secs = ctypes.c_double()
    L.oracle_alkane_run(ctypes.cast(arr, ctypes.c_void_p), n, steps, equilibration, seed, threads,
                        ctypes.cast(out, ctypes.c_void_p), ctypes.c_void_p(xyz.ctypes.data),
                        ctypes.c_void_p(ctypes.addressof(secs)), _ptr(xin), _ptr(nin))
    res = [out[i].as_dict() for i in range(n)]
    pos = []
    for i, q in enumerate(systems):
        nm = res[i]["n_molecules"]
        pos.append(xyz[offs[i]: offs[i] + nm * q.chain.n_beads * 3].reshape(nm, q.chain.n_beads, 3))
    del keep
    return res, pos, secs.value


def alkane_grow_vacuum(ff, chain, beta, n, seed=1, threads=0):
    """Chains grown in vacuum: (w[n], theta[n, nb-2], cos_phi[n, nb-3])."""
    L = _alkane_lib()
    o = off(ff)
    c = oalkane(chain, ff)
    nb = chain.n_beads
    w = np.empty(n)
    th = np.empty(n * max(0, nb - 2))
    cp = np.empty(n * max(0, nb - 3))
    L.oracle_alkane_grow_vacuum(ctypes.byref(o), ctypes.byref(c), beta, n, seed, threads, _ptr(w),
                                _ptr(th) if th.size else None, _ptr(cp) if cp.size else None)
    return w, th.reshape(n, max(0, nb - 2)), cp.reshape(n, max(0, nb - 3))


def alkane_energy(ff, system, xyz):
    """(framework-molecule VDW, molecule-molecule VDW, internal) of molecules xyz[n, nb, 3] in the system."""
    L = _alkane_lib()
    arr, keep = _alkane_setups(ff, [system])
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.empty(3)
    L.oracle_alkane_energy(ctypes.byref(arr[0]), _ptr(x), int(x.size // (3 * system.chain.n_beads)), _ptr(out))
    del keep
    return tuple(out)


def alkane_bead_energies(ff, system, xyz, beads, types, skip=-1):
    """Per-bead (framework, molecule, overlap) energies of single beads against the framework and molecules xyz."""
    L = _alkane_lib()
    arr, keep = _alkane_setups(ff, [system])
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
    b = np.ascontiguousarray(beads, dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(types, dtype=np.int32)
    n = len(t)
    fw, mm, ov = np.empty(n), np.empty(n), np.empty(n, dtype=np.int32)
    L.oracle_alkane_bead_energies(ctypes.byref(arr[0]), _ptr(x) if x.size else None,
                                  int(x.size // (3 * system.chain.n_beads)), _ptr(b), _ptr(t), n, skip, _ptr(fw),
                                  _ptr(mm), _ptr(ov))
    del keep
    return fw, mm, ov


# ---- mixture GCMC with identity change (oracle/mixture.cpp) ----
class OMixComponent(ctypes.Structure):
    _fields_ = [("n_atoms", ctypes.c_int32), ("starting_bead", ctypes.c_int32), ("offsets", ctypes.c_double * 24),
                ("masses", ctypes.c_double * 8), ("types", ctypes.c_int32 * 8), ("charges", ctypes.c_double * 8),
                ("fugacity", ctypes.c_double), ("w_ig", ctypes.c_double)]


class OMixSetup(ctypes.Structure):
    _fields_ = [("ff", ctypes.POINTER(OFF)), ("box", OBox), ("grid_cell", OBox), ("gnx", ctypes.c_int32),
                ("gny", ctypes.c_int32), ("gnz", ctypes.c_int32), ("grids", ctypes.c_void_p),
                ("s_framework", ctypes.c_void_p), ("n_components", ctypes.c_int32), ("comps", OMixComponent * 4),
                ("beta", ctypes.c_double), ("max_translation", ctypes.c_double), ("max_rotation", ctypes.c_double),
                ("p_translation", ctypes.c_double), ("p_rotation", ctypes.c_double), ("p_swap", ctypes.c_double),
                ("p_identity", ctypes.c_double), ("n_first_bead_trials", ctypes.c_int32),
                ("n_orientation_trials", ctypes.c_int32), ("max_molecules", ctypes.c_int32),
                ("use_ewald", ctypes.c_int32), ("framework", ctypes.c_void_p), ("n_framework", ctypes.c_int32)]


class OMixResult(ctypes.Structure):
    _fields_ = [("n_molecules", ctypes.c_int64 * 4), ("running_energy", ctypes.c_double),
                ("recomputed_energy", ctypes.c_double), ("sum_n", ctypes.c_double * 4), ("samples", ctypes.c_int64),
                ("attempted", ctypes.c_int64 * 5), ("accepted", ctypes.c_int64 * 5)]

    def as_dict(self):
        return {"n_molecules": list(self.n_molecules), "running_energy": self.running_energy,
                "recomputed_energy": self.recomputed_energy, "sum_n": list(self.sum_n), "samples": self.samples,
                "attempted": list(self.attempted), "accepted": list(self.accepted)}


def mixture_run(ff, cell, components, beta, fugacities, xyz, comp, steps, seed=1, grids=None, grid_dims=None,
                grid_cell=None, s_framework=None, use_ewald=True, max_translation=1.0,
                max_rotation=0.5235987755982988, probabilities=(1.0, 1.0, 1.0, 1.0), n_first=10, n_orient=10,
                max_molecules=512, w_ig=None, framework=None):
    """One oracle mixture run from the molecules xyz[n, na, 3] of components comp[n]; returns (result dict, final xyz,
    final comp, seconds). framework: atom records of the framework, seen explicitly by atom types without a grid."""
    L = lib()
    if not hasattr(L, "_mixture_declared"):
        L.oracle_mixture_run.argtypes = [ctypes.POINTER(OMixSetup), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]
        L._mixture_declared = True
    o = off(ff)
    s = OMixSetup()
    s.ff = ctypes.pointer(o)
    s.box = obox(cell)
    keep = [o]
    if grids is not None:
        arr = (ctypes.c_void_p * len(grids))()
        gk = [None if g is None else np.ascontiguousarray(g, dtype=np.float64) for g in grids]
        for i, g in enumerate(gk):
            arr[i] = None if g is None else g.ctypes.data
        keep += [arr, gk]
        s.grids = ctypes.cast(arr, ctypes.c_void_p)
        s.gnx, s.gny, s.gnz = grid_dims
        s.grid_cell = obox(grid_cell)
    if s_framework is not None:
        sf = np.ascontiguousarray(s_framework, dtype=np.float64)
        keep.append(sf)
        s.s_framework = sf.ctypes.data
    s.n_components = len(components)
    for k, comp_k in enumerate(components):
        c = s.comps[k]
        c.n_atoms = comp_k.n_atoms
        c.starting_bead = comp_k.starting_bead
        types, charges = comp_k.types(ff), comp_k.charges(ff)
        for i in range(comp_k.n_atoms):
            for d in range(3):
                c.offsets[3 * i + d] = float(comp_k.offsets[i][d])
            c.masses[i] = float(comp_k.masses[i])
            c.types[i] = int(types[i])
            c.charges[i] = float(charges[i])
        c.fugacity = fugacities[k]
        c.w_ig = 1.0 if w_ig is None else w_ig[k]
    s.beta = beta
    s.max_translation, s.max_rotation = max_translation, max_rotation
    s.p_translation, s.p_rotation, s.p_swap, s.p_identity = probabilities
    s.n_first_bead_trials, s.n_orientation_trials = n_first, n_orient
    s.max_molecules = max_molecules
    s.use_ewald = 1 if use_ewald else 0
    if framework is not None and len(framework):
        fw = np.ascontiguousarray(framework)
        keep.append(fw)
        s.framework, s.n_framework = fw.ctypes.data, len(fw)
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    cc = np.ascontiguousarray(comp, dtype=np.int32)
    na = components[0].n_atoms
    out = OMixResult()
    xo = np.zeros(max_molecules * na * 3)
    co = np.zeros(max_molecules, dtype=np.int32)
    secs = ctypes.c_double()
    L.oracle_mixture_run(ctypes.byref(s), _ptr(x) if len(cc) else None, _ptr(cc) if len(cc) else None, len(cc), steps,
                         seed, ctypes.c_void_p(ctypes.addressof(out)), _ptr(xo), _ptr(co),
                         ctypes.c_void_p(ctypes.addressof(secs)))
    r = out.as_dict()
    n = sum(r["n_molecules"])
    del keep
    return r, xo[: n * na * 3].reshape(n, na, 3), co[:n].copy(), secs.value

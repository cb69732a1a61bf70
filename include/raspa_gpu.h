/*
 * raspa_gpu.h — C-ABI of the B200 (sm_100a) implementation of RASPA3's data-parallel energy paths.
 *
 * Every entry point takes plain pointers and sizes and returns an rg_status. Host pointers stay owned by the
 * caller; device buffers passed in (out_device, ...) stay owned by the caller; buffers the library allocates
 * belong to the rg_ctx that allocated them and are freed by rg_ctx_destroy. One rg_ctx per host thread (or per
 * System): the library keeps no mutable global state besides the CUDA device context, so the calls are
 * re-entrant per context, matching the reference's one-System-per-thread drivers.
 *
 * A molecule overlap is a result (a flag in the output), never an error, as in the reference where it is a
 * std::nullopt. Units are the reference's internal units (energy 10 J/mol, length Angstrom, charge e).
 */
#ifndef RASPA_GPU_H
#define RASPA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t rg_status;
enum
{
  RG_OK = 0,
  RG_ERR_INVALID_ARGUMENT = 1,
  RG_ERR_CUDA = 2,
  RG_ERR_TIMEOUT = 3,
  RG_ERR_UNSUPPORTED = 4,
  RG_ERR_OUT_OF_MEMORY = 5,
  RG_ERR_NO_DEVICE = 6,
  RG_ERR_IO = 7,         /* a file could not be written or read */
  RG_ERR_CACHE_MISS = 8, /* rg_grid_load: no file, or one for other inputs, shape or a damaged one */
  RG_ERR_NONFINITE = 9   /* an input position, charge, scaling factor or cell entry is NaN or infinite: nothing is
                            launched (the reference has no such check; its sums would turn NaN) */
};

/* Byte-for-byte the reference Atom (src/raspakit/atom.ixx:28-39, 64 bytes): a std::span<const Atom> can be passed
 * as (const rg_atom*, size) without repacking. */
typedef struct rg_atom
{
  double x, y, z, w; /* double3 position (w: the union's padding lane, unused) */
  double charge;
  double scaling_vdw;
  double scaling_coulomb;
  uint32_t molecule_id;
  uint16_t type;
  uint8_t component_id;
  uint8_t group_fractional; /* low nibble: groupId (1-based dU/dlambda group, 0 = none); high nibble: isFractional */
} rg_atom;

/* SimulationBox (src/raspakit/simulationbox.ixx): cell[3*c + r] is component r of lattice vector c (the reference
 * double3x3 is column-major). triclinic != 0 selects the general minimum image. */
typedef struct rg_box
{
  double cell[9];
  int32_t triclinic;
} rg_box;

/* The ForceField fields these paths read (src/raspakit/forcefield/forcefield.ixx:88-174): the mixed, shifted
 * Lennard-Jones pair table (epsilon in internal units) and the cutoff / Ewald / overlap parameters. */
typedef struct rg_forcefield
{
  int32_t n_types;
  const double* epsilon; /* [n_types*n_types] */
  const double* sigma;   /* [n_types*n_types] */
  const double* shift;   /* [n_types*n_types] */
  const int32_t* lj;     /* [n_types*n_types] 1 = Lennard-Jones, 0 = None */
  double cutoff_framework_vdw;
  double cutoff_molecule_vdw;
  double cutoff_coulomb;
  double ewald_alpha;
  int32_t kmax_x, kmax_y, kmax_z;
  uint64_t recip_int_cutoff_sq; /* integer k-sphere bound; UINT64_MAX = full half-box */
  double recip_cutoff_sq;
  double overlap_criteria;
  int32_t use_charge;
  int32_t omit_inter;
} rg_forcefield;

typedef struct rg_ctx rg_ctx;
typedef struct rg_system rg_system; /* device-resident framework, grids, adsorbates and pair table of one system */
typedef struct rg_ewald rg_ewald;   /* device-resident k-vectors, prefactors and structure factors of one system */
typedef struct rg_mlp rg_mlp;       /* the learned proposal's network: parameters and optimizer state on the device */
typedef struct rg_proposal rg_proposal; /* a tabulated, exactly normalised first-bead proposal density */

/* ---- context ---- */
rg_status rg_ctx_create(int device, rg_ctx** out);
/* Objects created on a context (rg_system, rg_ewald, rg_gcmc) must be destroyed before it. */
rg_status rg_ctx_destroy(rg_ctx* ctx);
/* Use the caller's CUDA stream (a created cudaStream_t or cudaStreamPerThread; NULL restores the context's own
 * non-blocking stream, so the legacy NULL stream itself cannot be selected). */
rg_status rg_ctx_set_stream(rg_ctx* ctx, void* stream);
void* rg_ctx_stream(rg_ctx* ctx);
rg_status rg_ctx_synchronize(rg_ctx* ctx);
/* Message of the last failing call on this context ("" if none). */
const char* rg_ctx_last_error(rg_ctx* ctx);
const char* rg_version(void);

/* ---- (a) interpolation-grid build ---- */
enum
{
  RG_GRID_LENNARD_JONES = 0,
  RG_GRID_EWALD_REAL = 1, /* unit-charge real-space Ewald grid */
  RG_GRID_LENNARD_JONES_REPULSION = 2,
  RG_GRID_LENNARD_JONES_ATTRACTION = 3
};
enum
{
  RG_PRECISION_FP64 = 0,  /* FP64 pair terms and accumulation */
  RG_PRECISION_FP32C = 1  /* FP32 pair terms, compensated FP32 accumulation, FP64 epilogue */
};

/* Replaces InterpolationEnergyGrid::makeFrameworkInterpolationGrid, tricubic scheme
 * (src/raspakit/interpolation_energy_grid.cpp:3800-3978), with the per-point sums of
 * Interactions::calculateTricubicFractionalAtPosition (src/raspakit/interactions/framework_molecule_grid.cpp:168-282).
 * Called from System::createFrameworkInterpolationGrids (src/raspakit/system_interpolation_grids.cpp:211, 236).
 *
 * unit_atoms: the framework's unit-cell atoms (Cartesian, host memory); unit_cell: the framework unit cell;
 * cutoff: the cutoff that sizes the reference's supercell (cutOffFrameworkVDW for VDW grids, cutOffCoulomb for
 * the Ewald grid); the pair cutoff is ff->cutoff_framework_vdw, as in the reference. nx, ny, nz include the
 * duplicate periodic end-point. The result, 8 doubles per point in the reference layout
 * data[l + 8*(i + nx*(j + ny*k))], goes to out_device (a device buffer of 8*nx*ny*nz doubles) and/or out_host.
 * If stats is non-NULL it receives the work and traffic of the call; pair counting adds one integer add per pair. */
typedef struct rg_grid_stats
{
  int64_t pair_count;  /* in-cutoff pair evaluations (rr < rc^2, nonzero parameter): the algorithmic unit */
  int64_t n_images;    /* periodic images of the unit-cell atoms staged on the device */
  int64_t h2d_bytes;   /* host-to-device bytes copied by the call */
  int64_t d2h_bytes;   /* device-to-host bytes copied by the call */
} rg_grid_stats;

rg_status rg_grid_build(rg_ctx* ctx, int grid_type, const rg_forcefield* ff, const rg_box* unit_cell,
                        const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, double cutoff, int nx, int ny,
                        int nz, int precision, double* out_device, double* out_host, rg_grid_stats* stats);

/* Several grids of one framework in one call, replacing the grid loop of System::createFrameworkInterpolationGrids
 * (src/raspakit/system_interpolation_grids.cpp:202-238): grid g has type grid_types[g], probe probe_types[g] and goes
 * to the device buffer out_device[g] (8*nx*ny*nz doubles each) and, if out_host and out_host[g] are non-NULL, to that
 * host buffer too (the call then returns after the copies). Lennard-Jones grids whose probes see the same framework
 * atoms are computed two at a time in one pass over the candidate atoms. stats: n_grids entries or NULL. */
rg_status rg_grid_build_set(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell, const rg_atom* unit_atoms,
                            int n_unit_atoms, double cutoff, int nx, int ny, int nz, int precision, int n_grids,
                            const int* grid_types, const int* probe_types, double* const* out_device,
                            double* const* out_host, rg_grid_stats* stats);

/* Result of rg_grid_validate. sums[0..16]: the VDW term, sums[17..33]: the charge term (probe charge x unit-charge
 * Ewald grid), each as: sum w, sum w E_table, sum w E_full, sum w (E_full - E_table)^2, sum w E_full^2, then per axis
 * x, y, z: sum w G_table, sum w G_full, sum w (G_full - G_table)^2, sum w G_full^2 (energies in K, Cartesian gradients
 * in K/Angstrom, w = exp(-weight_beta * E_full,vdw)). The derived fields are the Boltzmann averages and the relative
 * errors sqrt(sum w diff^2 / sum w full^2) that the reference prints (NaN where a sum is zero). */
typedef struct rg_grid_validation
{
  int64_t n_points;        /* points tested */
  int64_t n_points_charge; /* points whose analytical VDW energy is below the overlap criterion (charge term) */
  double sums[34];
  double energy_table, energy_full, energy_relative_error;
  double gradient_table[3], gradient_full[3], gradient_relative_error[3];
  double charge_energy_table, charge_energy_full, charge_energy_relative_error;
  double charge_gradient_table[3], charge_gradient_full[3], charge_gradient_relative_error[3];
} rg_grid_validation;

/* The grid test of System::createFrameworkInterpolationGrids (src/raspakit/system_interpolation_grids.cpp:240-651,
 * tricubic scheme), which the reference runs serially after each grid build: at n_points points of the simulation
 * box, the interpolated energy and gradient of the VDW grid of probe_type (a device buffer laid out as rg_grid_build
 * writes it) against the analytical Lennard-Jones sum, and, with ewald_grid_device and a nonzero probe_charge, the
 * charge term against the analytical real-space Ewald sum where the VDW energy is below ff->overlap_criteria. The
 * points are `points` (3 fractions of the simulation box each, host memory) or, if NULL, drawn from `seed`.
 * weight_beta multiplies the energy in K in the Boltzmann weight: the reference uses System::beta (1/(kB T) in
 * inverse internal energy units) there; 1/T weights at temperature T. */
rg_status rg_grid_validate(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell, const rg_atom* unit_atoms,
                           int n_unit_atoms, const rg_box* simulation_box, int probe_type, int nx, int ny, int nz,
                           const double* vdw_grid_device, const double* ewald_grid_device, double probe_charge,
                           double weight_beta, int64_t n_points, uint64_t seed, const double* points,
                           rg_grid_validation* out);

/* Interpolation schemes (ForceField::InterpolationScheme, src/raspakit/forcefield/forcefield.ixx:79-84): the values
 * stored per grid point. */
enum
{
  RG_SCHEME_TRICUBIC = 8,    /* energy and its mixed first derivatives per cell axis (rg_grid_build) */
  RG_SCHEME_TRIQUINTIC = 27  /* all mixed derivatives up to second order per cell axis (rg_grid_build_triquintic) */
};
/* rg_grid_build_triquintic flags */
enum
{
  RG_TRIQUINTIC_REFERENCE_RECTANGULAR = 1, /* rectangular cells: keep the reference's two deviations (see below) */
  RG_TRIQUINTIC_FP32C = 2                  /* FP32 pair terms, compensated FP32 sums, FP64 epilogue (default FP64) */
};

/* Replaces the triquintic branch of InterpolationEnergyGrid::makeFrameworkInterpolationGrid
 * (src/raspakit/interpolation_energy_grid.cpp:3882-3962) with the per-point sums of
 * Interactions::calculateTriquinticFractionalAtPosition (src/raspakit/interactions/framework_molecule_grid.cpp:549-813).
 * Same arguments as rg_grid_build; FP64; grid_type RG_GRID_LENNARD_JONES or RG_GRID_EWALD_REAL (the reference's
 * triquintic branch evaluates the full Lennard-Jones factor for the repulsion and attraction types, which are
 * rejected with RG_ERR_UNSUPPORTED). The result, 27 doubles per point in the reference layout
 * data[l + 27*(i + nx*(j + ny*k))], channel l the mixed derivative of orders (ox, oy, oz) along the cell axes in the
 * reference order (0,0,0), (1,0,0), (0,1,0), (0,0,1), (2,0,0), (1,1,0), (1,0,1), (0,2,0), (0,1,1), (0,0,2), (2,1,0),
 * (2,0,1), (1,2,0), (1,1,1), (0,2,1), (1,0,2), (0,1,2), (2,2,0), (2,0,2), (0,2,2), (2,1,1), (1,2,1), (1,1,2), (2,2,1),
 * (2,1,2), (1,2,2), (2,2,2), goes to out_device (27*nx*ny*nz doubles) and/or out_host. The values are the exact
 * derivatives (those of the reference's triclinic branch for any cell). With RG_TRIQUINTIC_REFERENCE_RECTANGULAR a
 * rectangular cell gets the reference's rectangular branch instead, whose (0,1,0) and (0,0,1) channels are scaled by
 * cell[0][0] in place of cell[1][1] and cell[2][2] (framework_molecule_grid.cpp:648-650) and whose (2,2,2) channel
 * lacks its F3 term (:671-676). */
rg_status rg_grid_build_triquintic(rg_ctx* ctx, int grid_type, const rg_forcefield* ff, const rg_box* unit_cell,
                                   const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, double cutoff, int nx,
                                   int ny, int nz, int flags, double* out_device, double* out_host,
                                   rg_grid_stats* stats);

/* InterpolationEnergyGrid::interpolate and interpolateGradient (interpolation_energy_grid.cpp:3980-4178, 4211-4410,
 * tricubic and triquintic branches) on the device: the value and, if gradients is non-NULL, the Cartesian gradient
 * of a grid (a device buffer as rg_grid_build / rg_grid_build_triquintic write it, scheme RG_SCHEME_TRICUBIC or
 * RG_SCHEME_TRIQUINTIC) at n Cartesian positions (host, 3 doubles each). energies: n doubles; gradients: 3n. */
rg_status rg_grid_interpolate(rg_ctx* ctx, int scheme, const double* grid_device, int nx, int ny, int nz,
                              const rg_box* unit_cell, const double* positions, int n, double* energies,
                              double* gradients);

/* ---- grids on disk (host code; no device work) ----
 * The reference rebuilds every grid at start and restart: grids are not in its archive (system.cpp:1558-1562). These
 * calls keep a grid in a binary file keyed by a fingerprint of its inputs, so a restart can load it instead. */

/* 64-bit FNV-1a fingerprint of everything that determines a grid: grid type, scheme, flags, shape, unit cell, the
 * pair-table row of the probe (Lennard-Jones grids), cutoff, Ewald alpha, overlap criterion and the unit-cell atoms'
 * positions, charges and types. */
uint64_t rg_grid_fingerprint(int grid_type, int scheme, int flags, const rg_forcefield* ff, const rg_box* unit_cell,
                             const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, int nx, int ny, int nz);

/* Writes scheme*nx*ny*nz doubles (host memory, the layout rg_grid_build / rg_grid_build_triquintic write) with a header
 * (fingerprint, scheme, shape, cell, checksum of the values) to path, through a temporary file renamed into place. */
rg_status rg_grid_save(const char* path, uint64_t fingerprint, int scheme, const rg_box* unit_cell, int nx, int ny,
                       int nz, const double* data);

/* Reads a grid written by rg_grid_save into data (scheme*nx*ny*nz doubles) if the file exists and its fingerprint,
 * scheme, shape and checksum all match; RG_ERR_CACHE_MISS otherwise (data may then hold partial values). */
rg_status rg_grid_load(const char* path, uint64_t fingerprint, int scheme, int nx, int ny, int nz, double* data);

/* InterpolationEnergyGrid::writeOutput (interpolation_energy_grid.cpp:4760-4789): a cube file of the energy channel in
 * K, values in memory order (x fastest), one per line. The point counts are written as the negative numbers the
 * reference's cube reader expects (parseExternalFieldGridDimensions, :3516-3568); the reference's writer negates an
 * unsigned count there. origin: 3 doubles or NULL for (0, 0, 0).
 * unit_cell is the grid's own box (the framework unit cell the grid was built over), not the simulation box: the
 * header's voxel vectors are its cell vectors divided by the point counts. Only channel 0 (the energy) of a tricubic
 * or triquintic grid is written; a caller migrating from writeOutput(systemId, simulationBox, forceField) passes the
 * framework's unit cell. */
rg_status rg_grid_write_cube(const char* path, int scheme, const double* data, int nx, int ny, int nz,
                             const rg_box* unit_cell, const double* origin);

/* Hessian part of the triquintic grid test. sums[0..23]: the VDW term, sums[24..47]: the charge term; per term four
 * Boltzmann-weighted groups of six components (xx, xy, xz, yy, yz, zz): interpolated, analytical, squared difference,
 * squared analytical. The averages and relative errors follow from them as for the energy. */
typedef struct rg_grid_validation_hessian
{
  double sums[48];
  double hessian_table[6], hessian_full[6], hessian_relative_error[6];
  double charge_hessian_table[6], charge_hessian_full[6], charge_hessian_relative_error[6];
} rg_grid_validation_hessian;

/* The grid test of the triquintic scheme (system_interpolation_grids.cpp:240-760, triquintic branches): as
 * rg_grid_validate, with grids written by rg_grid_build_triquintic, the triquintic interpolant
 * (InterpolationEnergyGrid::interpolateHessian) and, in addition, the Hessians of both terms. The analytical side is
 * the exact derivative of the pair sums: for a rectangular non-cubic cell the reference's own rectangular branch
 * would report y and z gradients scaled by cell[0][0] (see rg_grid_build_triquintic). */
rg_status rg_grid_validate_triquintic(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell,
                                      const rg_atom* unit_atoms, int n_unit_atoms, const rg_box* simulation_box,
                                      int probe_type, int nx, int ny, int nz, const double* vdw_grid_device,
                                      const double* ewald_grid_device, double probe_charge, double weight_beta,
                                      int64_t n_points, uint64_t seed, const double* points, rg_grid_validation* out,
                                      rg_grid_validation_hessian* hessian);

/* Grid build that allocates nothing, for callers that cannot allocate device memory: applications whose device memory
 * is owned by another allocator (a host framework that reserves the whole device up front, or a memory pool with a hard
 * budget) where any cudaMalloc by a library would fail or break the budget. No counterpart in the reference.
 * Same arguments and result as rg_grid_build, minus the context: the caller passes the device, a stream (NULL = the
 * legacy default stream) and the device output buffer; there is no host output. The working memory is one fixed
 * file-scope device array that every GPU loading the library holds until exit; it holds at most 32768 periodic images
 * of the unit-cell atoms (RG_ERR_INVALID_ARGUMENT beyond that). The work runs with `device` current and the caller's
 * current device is restored before the call returns. All calls share the array: calls whose work overlaps on the GPU
 * (from several threads or streams) race; serialise them. */
rg_status rg_grid_build_noalloc(int device, void* stream, int grid_type, const rg_forcefield* ff,
                                const rg_box* unit_cell, const rg_atom* unit_atoms, int n_unit_atoms, int probe_type,
                                double cutoff, int nx, int ny, int nz, int precision, double* out_device,
                                rg_grid_stats* stats);

/* ---- (b) CBMC / CFCMC trial energies ---- */
/* External energy of one trial (the RunningEnergy fields of CBMC::FirstBeadTrial / ChainTrial), internal units. */
typedef struct rg_trial_energy
{
  double framework_vdw;
  double framework_charge;
  double molecule_vdw;
  double molecule_charge;
  double dudlambda_vdw[4];
  double dudlambda_charge[4];
  double external_field_vdw; /* RunningEnergy::externalFieldVDW of CBMC::computeExternalFieldEnergy */
  int32_t overlap; /* nonzero: the reference drops the trial (std::nullopt): 1 an overlap or a confining external
                      field's outside, 2 inside a blocked pocket */
  int32_t pad;
} rg_trial_energy;

/* A System's framework atoms (Cartesian, simulation-box frame), pair table and simulation box on ctx's device. */
rg_status rg_system_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* box, const rg_atom* framework_atoms,
                           int n_framework_atoms, rg_system** out);
rg_status rg_system_destroy(rg_system* system);
/* Attaches the tricubic grid of pseudo-atom `index` (index == ff->n_types: the unit-charge Ewald grid), the
 * System::interpolationGrids slots (src/raspakit/system.cpp:142). data: 8*nx*ny*nz doubles in the layout
 * rg_grid_build writes; data_on_device != 0 borrows a device buffer the caller keeps alive, else it is copied. */
rg_status rg_system_set_grid(rg_system* system, int index, const rg_box* unit_cell, int nx, int ny, int nz,
                             const double* data, int data_on_device);
/* Uploads the adsorbate atoms (System::spanOfMoleculeAtoms, the moleculeAtoms of CBMC::GrowContext). */
rg_status rg_system_set_molecules(rg_system* system, const rg_atom* atoms, int n_atoms);
/* Arithmetic of the trial energies and differences of this system: RG_PRECISION_FP64 (the default) or
 * RG_PRECISION_FP32C (Lennard-Jones pair terms in FP32 from the FP64 minimum-image displacement, TwoSum-compensated
 * FP32 sums per thread, FP64 totals; the real-space Coulomb pairs and the grid branch stay FP64, because charged
 * framework terms cancel by orders of magnitude and FP32 rounding of them would exceed 1e-6 of a trial's energy).
 * Both modes meet 1e-6 relative to each trial's energy. */
rg_status rg_system_set_precision(rg_system* system, int precision);

/* Interpolation scheme of this system's grids (ForceField::interpolationScheme): RG_SCHEME_TRICUBIC (the default,
 * 8 values per point) or RG_SCHEME_TRIQUINTIC (27, from rg_grid_build_triquintic). Set it before the first
 * rg_system_set_grid. rg_cbmc_external_energies, the energy differences and the device-resident Monte Carlo drivers
 * (rg_gcmc, rg_mixture, rg_proposal_sample_targets) then interpolate with that scheme (InterpolationEnergyGrid::
 * interpolate, interpolation_energy_grid.cpp:3980-4178). */
rg_status rg_system_set_interpolation_scheme(rg_system* system, int scheme);
/* Replaces CBMC::computeExternalNonOverlappingEnergies (src/raspakit/cbmc/interactions.cpp:54-179) and its callees
 * CBMC::insideBlockedPockets (:25-52), CBMC::computeExternalFieldEnergy (cbmc/interactions_external_field.cpp:22-200),
 * CBMC::computeFrameworkMoleculeEnergy (cbmc/interactions_framework_molecule.cpp:31-104) and
 * CBMC::computeInterMolecularEnergy (cbmc/interactions_intermolecular.cpp:22-95); called from the first-bead schemes
 * (cbmc/multiple_first_bead.cpp) and the chain growth (cbmc/flexible_molecules/insertion.cpp:63-64).
 * trials: n_trials consecutive sets of atoms_per_trial atoms (<= 64 per set, <= 4096 in total); skip: index within a
 * set to leave out (-1: none); skip_background_molecule: moleculeId of adsorbate atoms to leave out (-1: none).
 * out[t] gets trial t's energies; trials the reference drops are flagged (overlap != 0), not removed: an overlap, a
 * blocked pocket (rg_system_set_blocked_pockets) or an atom outside a confining external field
 * (rg_system_set_external_field). */
rg_status rg_cbmc_external_energies(rg_system* system, const rg_atom* trials, int n_trials, int atoms_per_trial,
                                    int skip, int64_t skip_background_molecule, double cutoff_framework_vdw,
                                    double cutoff_molecule_vdw, double cutoff_coulomb, rg_trial_energy* out);

/* CBMC::computeDualCutOffCorrection (src/raspakit/cbmc/interactions.cpp:214-251) with
 * computeExternalNonOverlappingEnergyDualCutOff (:181-212): the trial set's external energy with the force field's
 * cutoffs minus the same with dual_cutoff for all three, in one launch; out->overlap is nonzero where either is
 * dropped (the reference's std::nullopt). n_atoms <= 64. */
rg_status rg_cbmc_dual_cutoff_correction(rg_system* system, const rg_atom* trial_set, int n_atoms,
                                         int64_t skip_background_molecule, double dual_cutoff, rg_trial_energy* out);

/* ForceField::ChargeMethod (src/raspakit/forcefield/forcefield.ixx:31-39). This library implements the Ewald
 * real-space pair; the other methods are accepted where no charge term is evaluated (ff->use_charge == 0). */
enum
{
  RG_CHARGE_METHOD_EWALD = 0,
  RG_CHARGE_METHOD_COULOMB = 1,
  RG_CHARGE_METHOD_WOLF = 2,
  RG_CHARGE_METHOD_DAMPED_SHIFTED_FORCE = 3,
  RG_CHARGE_METHOD_MODIFIED_SHIFTED_FORCE = 4,
  RG_CHARGE_METHOD_ZERO_DIPOLE = 5
};

/* Replaces Interactions::computeFrameworkMoleculeEnergyDifference (src/raspakit/interactions/framework_molecule.cpp:
 * 117-252), called by the translation, rotation and CFCMC moves (mc_moves/component/translation.cpp:30-200,
 * rotation.cpp:30-190, swap_cfcmc.cpp): E(new atoms) - E(old atoms) against the framework of `system`. An atom takes
 * the grid branch only if it has a grid, is not fractional and charge_method is RG_CHARGE_METHOD_EWALD
 * (framework_molecule.cpp:145-146); otherwise the pair loop with the force field's cutoffs. out->overlap = 1 when a
 * new atom overlaps (the reference returns std::nullopt; old atoms are not tested). n_new, n_old <= 64. Other charge
 * methods with ff->use_charge set return RG_ERR_UNSUPPORTED. */
rg_status rg_framework_molecule_energy_difference(rg_system* system, int charge_method, const rg_atom* new_atoms,
                                                  int n_new, const rg_atom* old_atoms, int n_old, rg_trial_energy* out);

/* Replaces Interactions::computeInterMolecularEnergyDifference (src/raspakit/interactions/intermolecular.cpp:198-290),
 * called by the same moves: every adsorbate atom stored in `system` (rg_system_set_molecules) of another molecule
 * (moleculeId differs) against the new atoms minus against the old atoms, force-field cutoffs; zero when
 * ff->omit_inter is set. out->overlap = 1 when a new atom overlaps. n_new, n_old <= 64. */
rg_status rg_intermolecular_energy_difference(rg_system* system, const rg_atom* new_atoms, int n_new,
                                              const rg_atom* old_atoms, int n_old, rg_trial_energy* out);

/* Overwrites n_atoms stored adsorbate atoms from index first_atom on (the moved molecule's span after an accepted
 * move, as the reference copies the trial positions into System::spanOfMoleculeAtoms). */
rg_status rg_system_update_molecules(rg_system* system, int first_atom, const rg_atom* atoms, int n_atoms);

/* Component::blockingPockets for CBMC::insideBlockedPockets (src/raspakit/cbmc/interactions.cpp:25-52): 4 doubles per
 * pocket (centre as fractions of the framework unit cell, radius in Angstrom). A trial set with an atom closer than
 * radius * sqrt(scalingVDW) to a pocket centre (minimum image in the unit cell) is flagged 2 by
 * rg_cbmc_external_energies and rg_cbmc_dual_cutoff_correction. n_pockets = 0 clears the list. */
rg_status rg_system_set_blocked_pockets(rg_system* system, const rg_box* unit_cell, const double* pockets,
                                        int n_pockets);

/* ForceField::PotentialEnergySurfaceType (src/raspakit/forcefield/forcefield.ixx:50-68), the external field of
 * CBMC::computeExternalFieldEnergy. RG_SURFACE_OFF: no external field (System::hasExternalField false). */
enum
{
  RG_SURFACE_OFF = -1,
  RG_SURFACE_NONE = 0,
  RG_SURFACE_GRID_FILE = 1,
  RG_SURFACE_THIRD_ORDER_POLYNOMIAL = 3,
  RG_SURFACE_MULLER_BROWN = 8,
  RG_SURFACE_CYLINDER_X = 11,
  RG_SURFACE_CYLINDER_Y = 12,
  RG_SURFACE_CYLINDER_Z = 13,
  RG_SURFACE_RECTANGLE_X = 14,
  RG_SURFACE_RECTANGLE_Y = 15,
  RG_SURFACE_RECTANGLE_Z = 16
};
/* The external field of rg_cbmc_external_energies (cbmc/interactions_external_field.cpp:22-200). With `grid` (the
 * system's interpolation scheme, nx*ny*nz points over grid_box, the simulation box of
 * System::createExternalFieldInterpolationGrid; device memory the caller keeps alive if grid_on_device, else copied)
 * each atom adds scalingVDW times the interpolated value. Without a grid: the Muller-Brown surface, the x y z test
 * function, or a cylinder (radius geometry[0]) or rectangle (half-widths geometry[0], geometry[1]) along a cell axis
 * through the box centre whose outside drops the trial; the other surface types (0-16) add nothing, as in the
 * reference's switch. geometry: ForceField::externalFieldGeometryParameters (4 doubles, may be NULL). */
rg_status rg_system_set_external_field(rg_system* system, int surface_type, const double* geometry,
                                       const rg_box* grid_box, int nx, int ny, int nz, const double* grid,
                                       int grid_on_device);

/* ---- device-resident GCMC of a rigid component (many independent chains) ---- */
typedef struct rg_gcmc rg_gcmc;

/* A rigid component (Component, src/raspakit/component.ixx): body-frame positions relative to the centre of mass. */
typedef struct rg_gcmc_component
{
  int32_t n_atoms; /* <= 8 */
  int32_t starting_bead;
  int32_t types[8];
  double charges[8];
  double masses[8];
  double offsets[24];
} rg_gcmc_component;

typedef struct rg_gcmc_params
{
  double beta;     /* 1/(kB T), internal units (System::beta, system.cpp:98) */
  double fugacity; /* internal pressure units (pressure / PressureConversionFactor, system.cpp:96) */
  double cutoff_framework_vdw, cutoff_molecule_vdw, cutoff_coulomb;
  double max_translation; /* Angstrom, one Cartesian direction per move (translation.cpp:42-48) */
  double max_rotation;    /* radians, about one Cartesian axis (rotation.cpp:42-53) */
  double p_translation, p_rotation, p_swap; /* relative move probabilities; a swap is insertion or deletion 50/50 */
  int32_t n_first_bead_trials;              /* numberOfFirstBeadPositions (<= 16) */
  int32_t n_orientation_trials;             /* numberOfTrialDirections (<= 16) */
  int32_t max_molecules;                    /* molecules per chain */
  uint64_t seed;
} rg_gcmc_params;

typedef struct rg_gcmc_chain_result
{
  int64_t n_molecules;
  double energy; /* running total energy (framework + molecule-molecule + Ewald) */
  int64_t attempted[4], accepted[4]; /* translation, rotation, insertion, deletion */
  double sum_n, sum_n2, sum_energy;
  int64_t samples;
  double block_n[5]; /* loading averaged over 5 consecutive blocks of the recorded moves */
} rg_gcmc_chain_result;

/* n_chains independent GCMC chains of one rigid component in `system` (framework grids, pair table, simulation box),
 * each starting from an empty box; with charges, `ewald` (same box, rg_ewald_set_framework already called) provides
 * the k-vectors and the framework structure factor that every chain starts from. Moves: translation
 * (mc_moves/component/translation.cpp), rotation (rotation.cpp), CBMC insertion (insertion_cbmc.cpp:34-207) and
 * deletion (deletion_cbmc.cpp:34-195) with the first-bead and rigid-orientation trials of the reference's CBMC. */
rg_status rg_gcmc_create(rg_system* system, rg_ewald* ewald, const rg_gcmc_component* component,
                         const rg_gcmc_params* params, int n_chains, rg_gcmc** out);
rg_status rg_gcmc_destroy(rg_gcmc* gcmc);
/* Advances every chain by `moves` move attempts; record != 0 accumulates the statistics. Asynchronous on the ctx stream. */
rg_status rg_gcmc_run(rg_gcmc* gcmc, int64_t moves, int record);
rg_status rg_gcmc_results(rg_gcmc* gcmc, rg_gcmc_chain_result* out);
/* Positions (x, y, z per atom, molecules consecutive) of one chain, for recomputation checks. */
rg_status rg_gcmc_get_positions(rg_gcmc* gcmc, int chain, double* xyz, int capacity_atoms, int* n_molecules);

/* Uses a learned first-bead proposal for the CBMC insertion and deletion trials of every chain (NULL: back to uniform
 * positions). The trial weights become exp(-beta U) / q with q the proposal density relative to uniform; the
 * acceptance rules are unchanged, so the sampled ensemble is the same. The simulation box must be an integer
 * replication of unit_cell, the cell the proposal is defined on. No counterpart in the reference. */
rg_status rg_gcmc_set_proposal(rg_gcmc* gcmc, rg_proposal* proposal, const rg_box* unit_cell);

/* ---- learned first-bead proposal (no counterpart in the reference; plugs into the uniform first-bead sampling of
 * CBMC::growMoleculeMultipleFirstBeadSwapInsertion, src/raspakit/cbmc/multiple_first_bead.cpp:23-27) ---- */
/* A Fourier-feature MLP (96 inputs: sin, cos of 2 pi n s_a, n = 1..16, a = x, y, z; 2 SiLU layers of 64; 1 output,
 * 10,433 FP32 parameters) with He-uniform initial weights from `seed`. */
rg_status rg_mlp_create(rg_ctx* ctx, uint64_t seed, rg_mlp** out);
rg_status rg_mlp_destroy(rg_mlp* mlp);
int32_t rg_mlp_num_params(void);
/* Parameter vector order: W1 (64x96 row-major), b1, W2 (64x64), b2, w3 (64), b3. */
rg_status rg_mlp_get_params(rg_mlp* mlp, float* host, int32_t n);
rg_status rg_mlp_set_params(rg_mlp* mlp, const float* host, int32_t n);
/* Loss (1/n) sum (f(s_i) - t_i)^2 and its gradient over n samples (device arrays s: 3 per sample, t: 1). */
rg_status rg_mlp_loss_and_gradient(rg_mlp* mlp, const float* s_device, const float* target_device, int32_t n,
                                   float* loss, float* grad_host);
/* `steps` Adam steps on random minibatches of `batch` samples drawn from the n_samples device arrays. */
rg_status rg_mlp_train(rg_mlp* mlp, const float* s_device, const float* target_device, int64_t n_samples,
                       int32_t steps, int32_t batch, float learning_rate, uint64_t seed, float* final_loss);
/* f(s) for n fractional positions (device arrays). */
rg_status rg_mlp_evaluate(rg_mlp* mlp, const float* s_device, int64_t n, float* out_device);
/* Training data: n uniform fractional positions s of the unit cell and targets t = max(-beta U(s), t_min) with U the
 * framework energy of one bead of pseudo-atom type `pseudo_atom` and charge `charge` from the system's grids. */
rg_status rg_proposal_sample_targets(rg_system* system, int pseudo_atom, double charge, double beta, double t_min,
                                     const rg_box* unit_cell, int64_t n, uint64_t seed, float* s_device,
                                     float* t_device);
/* Tabulates exp(f) over cells_per_axis^3 cells of the unit cell into an exactly normalised density mixed with the
 * uniform density (weight eps_uniform > 0, so q > 0 everywhere). */
rg_status rg_proposal_create(rg_mlp* mlp, int32_t cells_per_axis, double eps_uniform, rg_proposal** out);
rg_status rg_proposal_destroy(rg_proposal* proposal);
/* The density relative to uniform at n fractional positions (host arrays, 3 per position). */
rg_status rg_proposal_density(rg_proposal* proposal, const double* s, int64_t n, double* q_out);

/* ---- (c) Ewald Fourier energy of a move ---- */
/* The Ewald part of RunningEnergy (src/raspakit/running_energy.ixx:500-540) in internal units. */
typedef struct rg_ewald_energy
{
  double ewald_fourier;
  double ewald_self;
  double ewald_exclusion;
  double dudlambda_ewald[4];
} rg_ewald_energy;

/* Builds the k-vector set of the box (kx in [0,kmax_x], ky, kz in [-kmax,kmax], k != 0, kx^2+ky^2+kz^2 <=
 * ff->recip_int_cutoff_sq, |k|^2 < ff->recip_cutoff_sq; ewald.cpp:1098-1146) and zeroed structure factors with
 * n_groups (0..4) dU/dlambda group sums. The state lives on ctx's device and stream. */
rg_status rg_ewald_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* box, int n_groups, rg_ewald** out);
rg_status rg_ewald_destroy(rg_ewald* ewald);
/* Number of k-vectors and the single-ion Fourier sum sum_k temp(k) (ewald.cpp:1146). */
rg_status rg_ewald_info(rg_ewald* ewald, int64_t* n_kvectors, double* single_ion_sum);
/* Replaces Interactions::precomputeEwaldFourierRigid (src/raspakit/interactions/ewald.cpp:276-348): the rigid
 * framework's structure factor, subtracted as a constant from every energy. */
rg_status rg_ewald_set_framework(rg_ewald* ewald, const rg_atom* framework_atoms, int n_framework_atoms);
/* Replaces Interactions::computeEwaldFourierEnergy (ewald.cpp:352-563): full recompute of the adsorbate structure
 * factors (stored), Fourier energy minus the framework-framework part, self, exclusion and net-charge terms.
 * molecule_sizes: atom counts of the consecutive molecules in atoms (for the intramolecular exclusion; counts that
 * are negative or add up to more than n_atoms give RG_ERR_INVALID_ARGUMENT). The host self, exclusion and net-charge
 * sums run while the structure-factor kernels are in flight. Called at initialisation, for drift checks and for volume
 * moves. */
rg_status rg_ewald_full(rg_ewald* ewald, const rg_atom* atoms, int n_atoms, const int32_t* molecule_sizes,
                        int n_molecules, double net_charge_framework, rg_ewald_energy* out);
/* Replaces Interactions::energyDifferenceEwaldFourier (ewald.cpp:1043-1244), called from every charged move
 * (e.g. mc_moves/component/translation.cpp, insertion_cbmc.cpp:99-101): the energy change of replacing old_atoms by
 * new_atoms (at most 512 together), leaving the trial structure factors on the device. net_charge: system net charge
 * before the move; net_charge_derivative_ext: 4 doubles or NULL (ewald.cpp:175-208). */
rg_status rg_ewald_delta(rg_ewald* ewald, const rg_atom* new_atoms, int n_new, const rg_atom* old_atoms, int n_old,
                         double net_charge, const double* net_charge_derivative_ext, rg_ewald_energy* out);
/* Replaces Interactions::acceptEwaldMove (ewald.cpp:1565-1574): the trial structure factors become the stored ones
 * (a pointer swap, no copy). */
rg_status rg_ewald_accept(rg_ewald* ewald);

/* ---- the structure-factor update of many systems at once ----
 * n_systems systems that share the box, force field and k-vectors of `ewald` (created without dU/dlambda groups),
 * each with its own stored and trial structure factors on the device: the Fourier part of
 * Interactions::energyDifferenceEwaldFourier (src/raspakit/interactions/ewald.cpp:1098-1162) for one move in every
 * system in one launch, and acceptEwaldMove (:1565-1574) per system as a buffer flip. It serves the drivers that
 * advance many independent systems (replicas, chains of a screening run); a system's self, exclusion and net-charge
 * terms need no structure factors and come from rg_ewald_delta's host terms (zero for translations and rotations).
 * Traffic per system and move: 32 bytes per k-vector (read S(k), write the trial S(k)). */
typedef struct rg_ewald_batch rg_ewald_batch;
rg_status rg_ewald_batch_create(rg_ewald* ewald, int n_systems, rg_ewald_batch** out);
rg_status rg_ewald_batch_destroy(rg_ewald_batch* batch);
/* Stored S(k) of one system: 2 nk doubles (re, im per k) from host memory, or, with sk == NULL, ewald's stored
 * structure factor (as rg_ewald_full or rg_ewald_set_structure_factors left it). */
rg_status rg_ewald_batch_set(rg_ewald_batch* batch, int system, const double* sk);
/* which = 0: the stored S(k) of a system, 1: its trial S(k) from the last rg_ewald_batch_delta (2 nk doubles). */
rg_status rg_ewald_batch_get(rg_ewald_batch* batch, int system, int which, double* sk);
/* One move per system: atoms[s * max_atoms ...] holds system s's n_new[s] new atoms followed by its n_old[s] old atoms
 * (at most 16 together). delta_fourier[s] receives the Fourier energy change (internal units, the ewald_fourier term
 * of rg_ewald_delta) and the system's trial S(k) is written. */
rg_status rg_ewald_batch_delta(rg_ewald_batch* batch, const rg_atom* atoms, int max_atoms, const int32_t* n_new,
                               const int32_t* n_old, double* delta_fourier);
/* accept[s] != 0: system s's trial S(k) becomes its stored S(k). */
rg_status rg_ewald_batch_accept(rg_ewald_batch* batch, const uint8_t* accept);
/* Device time of the last rg_ewald_batch_delta in milliseconds, from CUDA events on the context's stream: the upload
 * of the moved atoms and the update kernel (the host-side packing before them is not included). No reference
 * counterpart: it reports the kernel's duration for a roofline. Either pointer may be NULL. */
rg_status rg_ewald_batch_timing(rg_ewald_batch* batch, float* upload_ms, float* kernel_ms);
/* Copies structure factors to the host, 2*(1+n_groups) doubles per k-vector in the reference's storedEik order
 * (total, then group sums; re, im). which: 0 = stored, 1 = trial, 2 = framework (2 doubles per k). */
rg_status rg_ewald_get_structure_factors(rg_ewald* ewald, int which, double* host, int64_t n_doubles);
/* Overwrites the stored structure factors (e.g. from a restart file); n_doubles must equal 2*nk*(1+n_groups). */
rg_status rg_ewald_set_structure_factors(rg_ewald* ewald, const double* host, int64_t n_doubles);

/* ---- batched CBMC of flexible chains in many independent systems ---- */
/* A batch of independent systems of uneven size (framework atoms, chain length, trial counts), each running GCMC of
 * one flexible united-atom chain component with translation and CBMC swap moves. The whole batch advances in one
 * CUDA-graph replay of persistent kernels: one thread-block cluster per system keeps the system's framework atoms
 * (fixed-point fractional coordinates) and its molecules in shared memory for all moves of a launch. Replaces, per
 * system, the reference's CBMC::growFlexibleMoleculeChainInsertion (cbmc/flexible_molecules/insertion.cpp:32-126),
 * CBMC::retraceFlexibleMoleculeChainDeletion (deletion.cpp:30-104) with CBMC::generateGrowTrials /
 * generateRetraceTrials (cbmc/operators.cpp:951-1078) and the external energies of the trials
 * (CBMC::computeExternalNonOverlappingEnergies, cbmc/interactions.cpp:54-179), driven by
 * MC_Moves::insertionMoveCBMC / deletionMoveCBMC / translationMove. Pair terms are FP32 from exact fixed-point
 * displacements, reduced in FP64; Rosenbluth weights, acceptance and running energies are FP64. */
typedef struct rg_alkane rg_alkane;

/* A linear chain grown from bead 0 (Component with a fixed-bond / harmonic-bend / TraPPE-torsion definition). */
typedef struct rg_alkane_chain
{
  int32_t n_beads;              /* 2..8 */
  int32_t types[8];             /* pseudo-atom type of each bead */
  double bond_length;           /* BondType::Fixed, Angstrom */
  double bend_k, bend_theta0;   /* BendType::Harmonic 0.5 k (theta - theta0)^2: internal energy units, radians */
  double torsion[4];            /* TorsionType::TraPPE p0..p3, internal energy units */
  int32_t n_first_bead_trials;  /* 1..16 */
  int32_t n_trial_directions;   /* 1..16 (ForceField::numberOfTrialDirections) */
  int32_t n_torsion_trials;     /* 1..128 (ForceField::numberOfTorsionTrialDirections) */
  int32_t reserved;
} rg_alkane_chain;

typedef struct rg_alkane_system
{
  rg_box box;                   /* simulation box (already replicated for the minimum image of the cutoffs) */
  const rg_atom* framework;     /* framework atoms of the simulation box, Cartesian */
  int32_t n_framework;
  int32_t max_molecules;        /* 1..256 */
  rg_alkane_chain chain;
  double beta, fugacity;        /* 1/(kB T) and fugacity, internal units */
  double w_ig;                  /* ideal-gas Rosenbluth weight (Component::idealGasRosenbluthWeight) */
  double max_translation;       /* Angstrom */
  double p_translation, p_swap; /* relative move probabilities */
} rg_alkane_system;

/* The launch plan: systems sorted by work; the first `split` run as clusters of cluster_big CTAs, the rest as
 * clusters of cluster_small; `threads` per CTA; `moves_per_launch` moves per persistent launch. */
typedef struct rg_alkane_plan
{
  int32_t cluster_big, cluster_small, threads, split, moves_per_launch, reserved;
  double ms_per_move; /* measured by rg_alkane_autotune (device time per move of every system) */
} rg_alkane_plan;

/* Uploads the batch; every system starts empty. Pair parameters come from ff (mixed, shifted Lennard-Jones; the
 * framework and molecule VDW cutoffs and the overlap criterion). Framework atoms whose type has no Lennard-Jones
 * interaction with any bead type are dropped (they contribute nothing). */
rg_status rg_alkane_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_alkane_system* systems, int n_systems,
                           uint64_t seed, rg_alkane** out);
rg_status rg_alkane_destroy(rg_alkane* batch);
/* Times candidate plans on the batch (cluster sizes 1/2/4 per class, 128/256/512 threads; each from the same snapshot
 * of the state, restored afterwards so tuning does not advance the simulation), keeps the fastest and returns it in
 * *chosen (may be NULL). */
rg_status rg_alkane_autotune(rg_alkane* batch, int moves_per_candidate, rg_alkane_plan* chosen);
rg_status rg_alkane_set_plan(rg_alkane* batch, const rg_alkane_plan* plan);
rg_status rg_alkane_get_plan(rg_alkane* batch, rg_alkane_plan* plan);
/* Advances every system by `moves` move attempts (graph replays on the context stream); record != 0 accumulates the
 * statistics returned by rg_alkane_results. Asynchronous: returns once the work is enqueued. */
rg_status rg_alkane_run(rg_alkane* batch, int64_t moves, int record);
/* Per-system statistics (attempted/accepted [0] translation, [2] insertion, [3] deletion) and running energy. */
rg_status rg_alkane_results(rg_alkane* batch, rg_gcmc_chain_result* out);
/* Positions of system s: n_molecules * n_beads * 3 doubles (Cartesian, each molecule unwrapped). */
rg_status rg_alkane_get_positions(rg_alkane* batch, int system, double* xyz, int capacity_doubles, int* n_molecules);
/* Replaces the molecules of system s (e.g. a restart) and its running energy. */
rg_status rg_alkane_set_positions(rg_alkane* batch, int system, const double* xyz, int n_molecules, double energy);
/* External energies of single beads in system s against its framework and molecules (skipping molecule `skip`, or
 * -1): the trial-energy kernel of the batch on one system, the counterpart of
 * CBMC::computeExternalNonOverlappingEnergies for single-bead trials. fw, mm: per-bead energies; overlap: 1 where a
 * pair exceeds the overlap criterion. n_beads <= 16. */
rg_status rg_alkane_bead_energies(rg_alkane* batch, int system, const double* xyz_beads, const int32_t* types,
                                  int n_beads, int skip, double* fw, double* mm, int32_t* overlap);
/* In-cutoff pair evaluations (trial bead x framework atom or molecule bead with r < rc) since creation, summed
 * over the systems: the algorithmic unit of the trial energies. */
rg_status rg_alkane_pair_count(rg_alkane* batch, uint64_t* total);
/* Monte Carlo kernel launches enqueued by this batch so far (each kernel node of a graph replay counts once). */
rg_status rg_alkane_launch_count(rg_alkane* batch, int64_t* launches);
/* Grows n chains in vacuum on the device: the ideal-gas Rosenbluth weight <W> (*w_mean; the W_IG of the acceptance
 * rule) and optionally per chain w[n], the bend angles theta[n*(nb-2)] and torsion cosines cos_phi[n*(nb-3)]. */
rg_status rg_alkane_grow_vacuum(rg_ctx* ctx, const rg_forcefield* ff, const rg_alkane_chain* chain, double beta,
                                int64_t n, uint64_t seed, double* w_mean, double* w, double* theta, double* cos_phi);

/* ---- one large system of several rigid components on the whole GPU ---- */
/* GCMC of a mixture in one system: translation, rotation, CBMC insertion / deletion and identity change
 * (mc_moves/component/translation.cpp, rotation.cpp, insertion_cbmc.cpp, deletion_cbmc.cpp, identity_change.cpp). Every
 * move runs on all SMs: molecule sites and k-vectors are split between the CTAs of one cooperative persistent kernel,
 * which meet at a grid barrier once per phase (one phase per move, two for an insertion). Framework energies come from
 * the grids of `system`, molecule-molecule pairs are FP32 from exact fixed-point displacements with FP64 sums, the
 * Fourier part uses `ewald`'s k-vectors (FP64). */
typedef struct rg_mixture rg_mixture;

typedef struct rg_mixture_params
{
  double beta;
  double fugacity[4];     /* per component, internal units */
  double w_ig[4];         /* ideal-gas Rosenbluth weight per component (0 = 1) */
  double cutoff_molecule_vdw, cutoff_coulomb;
  double cutoff_framework_vdw; /* explicit framework pairs of atom types without a VDW grid */
  double max_translation, max_rotation;
  double p_translation, p_rotation, p_swap, p_identity; /* a component is chosen uniformly, then the move */
  int32_t n_first_bead_trials, n_orientation_trials;    /* 1..12 */
  int32_t max_molecules;
  int32_t n_blocks;       /* CTAs of the cooperative launch (0: one per SM) */
  uint64_t seed;
} rg_mixture_params;

typedef struct rg_mixture_result
{
  int64_t n_molecules[4];
  double energy;                     /* running total energy */
  int64_t attempted[5], accepted[5]; /* translation, rotation, insertion, deletion, identity change */
  double sum_n[4];                   /* sum over recorded moves of each component's count */
  double sum_energy;
  int64_t samples;
  int32_t status;                    /* RG_OK, or RG_ERR_TIMEOUT if a grid barrier gave up */
  int32_t reserved;
} rg_mixture_result;

/* components: all with the same atom count (2-4); the starting configuration is n_molecules molecules at xyz
 * (n_atoms * 3 doubles each) of components comp_of_molecule. Set the running energy and the structure factors of
 * that configuration with rg_mixture_set_state before running. */
rg_status rg_mixture_create(rg_system* system, rg_ewald* ewald, const rg_gcmc_component* components, int n_components,
                            const rg_mixture_params* params, const double* xyz, const int32_t* comp_of_molecule,
                            int n_molecules, rg_mixture** out);
/* Frees the mixture's device state (destroy it before its system, Ewald state and context). */
rg_status rg_mixture_destroy(rg_mixture* mixture);
/* energy: total energy of the configuration; sk: its structure factors (framework included), 2 doubles per k-vector
 * in the rg_ewald order (NULL: leave them). */
rg_status rg_mixture_set_state(rg_mixture* mixture, double energy, const double* sk, int64_t n_doubles);
/* Advances the system by `moves` move attempts (the mix of mc_moves/mc_moves.cpp's component moves); record != 0
 * accumulates the loading and energy averages. Results, positions and structure factors are read afterwards. */
rg_status rg_mixture_run(rg_mixture* mixture, int64_t moves, int record);
/* Several independent mixtures advanced by one cooperative launch: system s runs on CTAs [s B, (s + 1) B), B the
 * CTA count every one of them was created with (rg_mixture_params.n_blocks, the same for all), so n systems share the
 * GPU instead of each leaving most SMs idle. All on one rg_ctx, created from the same system, Ewald state, components
 * and parameters (they may differ in their molecules and seeds; RG_ERR_INVALID_ARGUMENT otherwise); n <= 148 and n B
 * CTAs must fit on the GPU at once (one CTA per SM). Fewer CTAs per system give more aggregate moves per second as
 * long as a system's k-vectors fit (at kmax 12, 2 CTAs). No counterpart in the reference, whose systems run on
 * separate threads. */
rg_status rg_mixture_run_many(rg_mixture* const* mixtures, int n, int64_t moves, int record);
rg_status rg_mixture_results(rg_mixture* mixture, rg_mixture_result* out);
/* Test of the bounded grid-barrier wait (no counterpart in the reference, whose moves run on one CPU thread): in the
 * next launch CTA absent_cta does not arrive at the first barrier, so every CTA's wait gives up after spin_limit polls
 * (at most the production limit), the launch raises its error flag and leaves, rg_mixture_results reports
 * RG_ERR_TIMEOUT, and later launches return without doing anything; the mixture must then be destroyed. absent_cta
 * = -1 arrives normally. Nothing faults or hangs: the wait ends by itself. */
rg_status rg_mixture_set_wait_test(rg_mixture* mixture, int absent_cta, int64_t spin_limit);
/* The current molecules, made whole (n_atoms * 3 doubles each) with their components, for output or a restart;
 * capacity_molecules bounds what xyz and comp can hold, *n_molecules receives the count. */
rg_status rg_mixture_get_positions(rg_mixture* mixture, double* xyz, int32_t* comp, int capacity_molecules,
                                   int* n_molecules);
/* The current structure factors (framework included), 2 doubles per k-vector in the rg_ewald order: storedEik. */
rg_status rg_mixture_get_structure_factors(rg_mixture* mixture, double* host, int64_t n_doubles);
/* Learned first-bead proposal of one component (NULL: uniform). */
rg_status rg_mixture_set_proposal(rg_mixture* mixture, int component, rg_proposal* proposal, const rg_box* unit_cell);
rg_status rg_mixture_info(rg_mixture* mixture, int* blocks, int64_t* nk);

/* ---- measurement ---- */
/* FP32 (precision = RG_PRECISION_FP32C) or FP64 FMA throughput of this device in TFLOP/s, from independent FMA chains
 * on every SM: the SIMT-pipe denominator for the pair kernels' rooflines. No counterpart in the reference. */
rg_status rg_probe_fma_peak(rg_ctx* ctx, int precision, double* tflops, double* seconds);

#ifdef __cplusplus
}
#endif

#endif

// raspa_b200.hpp — C++20 host layer over the C-ABI (include/raspa_gpu.h), mirroring the RASPA3 interface of the paths
// it replaces: the same names, the same argument meaning and the same error behaviour (a precondition failure throws
// std::runtime_error; a trial overlap drops the trial, as the reference's std::nullopt does).
//
//   InterpolationEnergyGrid::makeFrameworkInterpolationGrid   src/raspakit/interpolation_energy_grid.cpp:3800-3978
//   Interactions::computeEwaldFourierEnergy                   src/raspakit/interactions/ewald.cpp:352-563
//   Interactions::energyDifferenceEwaldFourier                src/raspakit/interactions/ewald.cpp:1043-1244
//   Interactions::acceptEwaldMove                             src/raspakit/interactions/ewald.cpp:1565-1574
//   CBMC::computeExternalNonOverlappingEnergies               src/raspakit/cbmc/interactions.cpp:54-132
//
// Header-only; link against libraspagpu.so. Types are those of the C-ABI (rg_atom is layout-identical to the
// reference Atom, so a std::span<const Atom> can be reinterpreted as std::span<const rg_atom>).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/raspa_gpu.h"

namespace raspa_b200
{
inline void check(rg_ctx* ctx, rg_status st, const char* what)
{
  if (st != RG_OK)
    throw std::runtime_error(std::string("[raspa_b200] ") + what + " failed (status " + std::to_string(st) +
                             "): " + (ctx ? rg_ctx_last_error(ctx) : ""));
}

// One device context (stream + scratch) per host thread / System.
class Context
{
 public:
  explicit Context(int device = 0) { check(nullptr, rg_ctx_create(device, &ctx_), "rg_ctx_create"); }
  ~Context() { rg_ctx_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  rg_ctx* get() const { return ctx_; }

 private:
  rg_ctx* ctx_ = nullptr;
};

// The ForceField fields these paths read; owns the mixed pair table.
struct ForceField
{
  int32_t numberOfPseudoAtoms = 0;
  std::vector<double> epsilon, sigma, shift;  // [n*n], epsilon in internal units
  std::vector<int32_t> lj;                    // [n*n]
  double cutOffFrameworkVDW = 12.0, cutOffMoleculeVDW = 12.0, cutOffCoulomb = 12.0;
  double EwaldAlpha = 0.265058;
  std::array<int32_t, 3> numberOfWaveVectors{8, 8, 8};
  uint64_t reciprocalIntegerCutOffSquared = UINT64_MAX;
  double reciprocalCutOffSquared = 1.7976931348623157e308;
  double energyOverlapCriteria = 1e6;
  int chargeMethod = RG_CHARGE_METHOD_EWALD;  // ForceField::chargeMethod
  bool useCharge = true;
  bool omitInterInteractions = false;

  rg_forcefield abi() const
  {
    rg_forcefield f{};
    f.n_types = numberOfPseudoAtoms;
    f.epsilon = epsilon.data();
    f.sigma = sigma.data();
    f.shift = shift.data();
    f.lj = lj.data();
    f.cutoff_framework_vdw = cutOffFrameworkVDW;
    f.cutoff_molecule_vdw = cutOffMoleculeVDW;
    f.cutoff_coulomb = cutOffCoulomb;
    f.ewald_alpha = EwaldAlpha;
    f.kmax_x = numberOfWaveVectors[0];
    f.kmax_y = numberOfWaveVectors[1];
    f.kmax_z = numberOfWaveVectors[2];
    f.recip_int_cutoff_sq = reciprocalIntegerCutOffSquared;
    f.recip_cutoff_sq = reciprocalCutOffSquared;
    f.overlap_criteria = energyOverlapCriteria;
    f.use_charge = useCharge ? 1 : 0;
    f.omit_inter = omitInterInteractions ? 1 : 0;
    return f;
  }
};

// SimulationBox: columns of `cell` are the lattice vectors.
inline rg_box makeBox(const std::array<std::array<double, 3>, 3>& columns)
{
  rg_box b{};
  bool tri = false;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
    {
      b.cell[3 * c + r] = columns[c][r];
      if (c != r && columns[c][r] != 0.0) tri = true;
    }
  b.triclinic = tri ? 1 : 0;
  return b;
}

// RunningEnergy fields these paths produce (internal units).
struct RunningEnergy
{
  double externalFieldVDW = 0;
  double frameworkMoleculeVDW = 0, frameworkMoleculeCharge = 0, moleculeMoleculeVDW = 0, moleculeMoleculeCharge = 0;
  double ewald_fourier = 0, ewald_self = 0, ewald_exclusion = 0;
  std::array<double, 4> dudlambdaVDW{}, dudlambdaCharge{}, dudlambdaEwald{};
  double ewaldFourier() const { return ewald_fourier + ewald_self + ewald_exclusion; }
  double potentialEnergy() const
  {
    return externalFieldVDW + frameworkMoleculeVDW + frameworkMoleculeCharge + moleculeMoleculeVDW +
           moleculeMoleculeCharge + ewald_fourier + ewald_self + ewald_exclusion;
  }
};

enum class InterpolationGridType : int
{
  LennardJones = RG_GRID_LENNARD_JONES,
  EwaldReal = RG_GRID_EWALD_REAL,
  LennardJonesRepulsion = RG_GRID_LENNARD_JONES_REPULSION,
  LennardJonesAttraction = RG_GRID_LENNARD_JONES_ATTRACTION
};

// ForceField::InterpolationScheme values this layer builds (forcefield/forcefield.ixx:79-84)
enum class InterpolationScheme : int
{
  Tricubic = RG_SCHEME_TRICUBIC,
  Triquintic = RG_SCHEME_TRIQUINTIC
};

// InterpolationEnergyGrid (src/raspakit/interpolation_energy_grid.ixx): `order` doubles per point (8 tricubic, 27
// triquintic) in the reference layout.
class InterpolationEnergyGrid
{
 public:
  InterpolationEnergyGrid(const rg_box& unitCellBox, std::array<int, 3> numberOfGridPoints,
                          InterpolationScheme order = InterpolationScheme::Tricubic)
      : unitCellBox(unitCellBox),
        numberOfGridPoints(numberOfGridPoints),
        order(order),
        data(static_cast<size_t>(order) * static_cast<size_t>(numberOfGridPoints[0]) * numberOfGridPoints[1] *
             numberOfGridPoints[2])
  {
  }

  // precision: RG_PRECISION_FP64 or RG_PRECISION_FP32C (tricubic); the triquintic build takes
  // RG_TRIQUINTIC_FP32C for FP32C and keeps the exact derivatives unless referenceRectangular is set
  void makeFrameworkInterpolationGrid(Context& ctx, InterpolationGridType interpolationGridType,
                                      const ForceField& forceField, std::span<const rg_atom> frameworkUnitCellAtoms,
                                      double cutOff, std::size_t pseudo_atom_index,
                                      int precision = RG_PRECISION_FP64, bool referenceRectangular = false)
  {
    const rg_forcefield f = forceField.abi();
    if (order == InterpolationScheme::Triquintic)
    {
      const int flags = (referenceRectangular ? RG_TRIQUINTIC_REFERENCE_RECTANGULAR : 0) |
                        (precision == RG_PRECISION_FP32C ? RG_TRIQUINTIC_FP32C : 0);
      check(ctx.get(),
            rg_grid_build_triquintic(ctx.get(), static_cast<int>(interpolationGridType), &f, &unitCellBox,
                                     frameworkUnitCellAtoms.data(), static_cast<int>(frameworkUnitCellAtoms.size()),
                                     static_cast<int>(pseudo_atom_index), cutOff, numberOfGridPoints[0],
                                     numberOfGridPoints[1], numberOfGridPoints[2], flags, nullptr, data.data(),
                                     nullptr),
            "makeFrameworkInterpolationGrid");
      return;
    }
    check(ctx.get(),
          rg_grid_build(ctx.get(), static_cast<int>(interpolationGridType), &f, &unitCellBox,
                        frameworkUnitCellAtoms.data(), static_cast<int>(frameworkUnitCellAtoms.size()),
                        static_cast<int>(pseudo_atom_index), cutOff, numberOfGridPoints[0], numberOfGridPoints[1],
                        numberOfGridPoints[2], precision, nullptr, data.data(), nullptr),
          "makeFrameworkInterpolationGrid");
  }

  // InterpolationEnergyGrid::writeOutput (interpolation_energy_grid.cpp:4760-4789): the energy channel as a cube file
  void writeOutput(const std::string& path, std::array<double, 3> origin = {0.0, 0.0, 0.0}) const
  {
    check(nullptr,
          rg_grid_write_cube(path.c_str(), static_cast<int>(order), data.data(), numberOfGridPoints[0],
                             numberOfGridPoints[1], numberOfGridPoints[2], &unitCellBox, origin.data()),
          "writeOutput");
  }

  rg_box unitCellBox;
  std::array<int, 3> numberOfGridPoints;
  InterpolationScheme order;
  std::vector<double> data;
};

namespace Interactions
{
// The device-resident storedEik / trialEik / fixedFrameworkStoredEik of one System.
class EwaldState
{
 public:
  EwaldState(Context& ctx, const ForceField& forceField, const rg_box& simulationBox, int groups = 0) : ctx_(&ctx)
  {
    const rg_forcefield f = forceField.abi();
    check(ctx.get(), rg_ewald_create(ctx.get(), &f, &simulationBox, groups, &e_), "rg_ewald_create");
  }
  ~EwaldState() { rg_ewald_destroy(e_); }
  EwaldState(const EwaldState&) = delete;
  EwaldState& operator=(const EwaldState&) = delete;
  rg_ewald* get() const { return e_; }
  rg_ctx* ctx() const { return ctx_->get(); }
  double singleIonFourierSum() const
  {
    double s = 0.0;
    rg_ewald_info(e_, nullptr, &s);
    return s;
  }

 private:
  Context* ctx_;
  rg_ewald* e_ = nullptr;
};

inline RunningEnergy fromEwald(const rg_ewald_energy& e)
{
  RunningEnergy r;
  r.ewald_fourier = e.ewald_fourier;
  r.ewald_self = e.ewald_self;
  r.ewald_exclusion = e.ewald_exclusion;
  for (int g = 0; g < 4; ++g) r.dudlambdaEwald[g] = e.dudlambda_ewald[g];
  return r;
}

// precomputeEwaldFourierRigid (ewald.cpp:276-348)
inline void precomputeEwaldFourierRigid(EwaldState& state, std::span<const rg_atom> rigidFrameworkAtoms)
{
  check(state.ctx(),
        rg_ewald_set_framework(state.get(), rigidFrameworkAtoms.data(), static_cast<int>(rigidFrameworkAtoms.size())),
        "precomputeEwaldFourierRigid");
}

// computeEwaldFourierEnergy (ewald.cpp:352-563)
inline RunningEnergy computeEwaldFourierEnergy(EwaldState& state, std::span<const rg_atom> moleculeAtomPositions,
                                               std::span<const int32_t> moleculeSizes, double netChargeFramework = 0.0)
{
  rg_ewald_energy e{};
  check(state.ctx(),
        rg_ewald_full(state.get(), moleculeAtomPositions.data(), static_cast<int>(moleculeAtomPositions.size()),
                      moleculeSizes.data(), static_cast<int>(moleculeSizes.size()), netChargeFramework, &e),
        "computeEwaldFourierEnergy");
  return fromEwald(e);
}

// energyDifferenceEwaldFourier (ewald.cpp:1043-1244): leaves trialEik on the device
inline RunningEnergy energyDifferenceEwaldFourier(EwaldState& state, std::span<const rg_atom> newatoms,
                                                  std::span<const rg_atom> oldatoms, double netCharge = 0.0)
{
  rg_ewald_energy e{};
  check(state.ctx(),
        rg_ewald_delta(state.get(), newatoms.data(), static_cast<int>(newatoms.size()), oldatoms.data(),
                       static_cast<int>(oldatoms.size()), netCharge, nullptr, &e),
        "energyDifferenceEwaldFourier");
  return fromEwald(e);
}

// acceptEwaldMove (ewald.cpp:1565-1574)
inline void acceptEwaldMove(EwaldState& state) { check(state.ctx(), rg_ewald_accept(state.get()), "acceptEwaldMove"); }
}  // namespace Interactions

namespace CBMC
{
// The device-resident data of CBMC::GrowContext (cbmc/cbmc_growth_context.ixx:13-27).
class GrowContext
{
 public:
  GrowContext(Context& ctx, const ForceField& forceField, const rg_box& simulationBox,
              std::span<const rg_atom> frameworkAtoms)
      : ctx_(&ctx), forceField_(forceField)
  {
    const rg_forcefield f = forceField.abi();
    check(ctx.get(),
          rg_system_create(ctx.get(), &f, &simulationBox, frameworkAtoms.data(),
                           static_cast<int>(frameworkAtoms.size()), &s_),
          "rg_system_create");
  }
  ~GrowContext() { rg_system_destroy(s_); }
  GrowContext(const GrowContext&) = delete;
  GrowContext& operator=(const GrowContext&) = delete;

  void setInterpolationGrid(std::size_t index, const InterpolationEnergyGrid& grid)
  {
    check(ctx_->get(),
          rg_system_set_grid(s_, static_cast<int>(index), &grid.unitCellBox, grid.numberOfGridPoints[0],
                             grid.numberOfGridPoints[1], grid.numberOfGridPoints[2], grid.data.data(), 0),
          "rg_system_set_grid");
  }
  void setMoleculeAtoms(std::span<const rg_atom> moleculeAtoms)
  {
    check(ctx_->get(), rg_system_set_molecules(s_, moleculeAtoms.data(), static_cast<int>(moleculeAtoms.size())),
          "rg_system_set_molecules");
  }
  // an accepted move: the molecule's atoms from index `first` on, as the reference copies them into
  // System::spanOfMoleculeAtoms
  void updateMoleculeAtoms(std::size_t first, std::span<const rg_atom> atoms)
  {
    check(ctx_->get(),
          rg_system_update_molecules(s_, static_cast<int>(first), atoms.data(), static_cast<int>(atoms.size())),
          "rg_system_update_molecules");
  }
  // Component::blockingPockets: {fractional x, y, z, radius} in the framework's unit cell
  void setBlockedPockets(const rg_box& frameworkUnitCell, const std::vector<std::array<double, 4>>& pockets)
  {
    check(ctx_->get(),
          rg_system_set_blocked_pockets(s_, &frameworkUnitCell, pockets.empty() ? nullptr : pockets.front().data(),
                                        static_cast<int>(pockets.size())),
          "rg_system_set_blocked_pockets");
  }
  // System::hasExternalField with ForceField::potentialEnergySurfaceType / externalFieldGeometryParameters, or the
  // external-field grid over the simulation box (RG_SURFACE_OFF switches it off)
  void setExternalField(int surfaceType, const std::array<double, 4>& geometry,
                        const InterpolationEnergyGrid* grid = nullptr)
  {
    check(ctx_->get(),
          rg_system_set_external_field(s_, surfaceType, geometry.data(), grid ? &grid->unitCellBox : nullptr,
                                       grid ? grid->numberOfGridPoints[0] : 0, grid ? grid->numberOfGridPoints[1] : 0,
                                       grid ? grid->numberOfGridPoints[2] : 0, grid ? grid->data.data() : nullptr, 0),
          "rg_system_set_external_field");
  }
  rg_system* get() const { return s_; }
  rg_ctx* ctx() const { return ctx_->get(); }
  const ForceField& forceField() const { return forceField_; }

 private:
  Context* ctx_;
  const ForceField& forceField_;
  rg_system* s_ = nullptr;
};

struct FirstBeadTrial
{
  rg_atom position;
  RunningEnergy energy;
};

struct ChainTrial
{
  std::vector<rg_atom> positions;
  RunningEnergy energy;
};

inline RunningEnergy fromTrial(const rg_trial_energy& t)
{
  RunningEnergy r;
  r.externalFieldVDW = t.external_field_vdw;
  r.frameworkMoleculeVDW = t.framework_vdw;
  r.frameworkMoleculeCharge = t.framework_charge;
  r.moleculeMoleculeVDW = t.molecule_vdw;
  r.moleculeMoleculeCharge = t.molecule_charge;
  for (int g = 0; g < 4; ++g)
  {
    r.dudlambdaVDW[g] = t.dudlambda_vdw[g];
    r.dudlambdaCharge[g] = t.dudlambda_charge[g];
  }
  return r;
}

// computeExternalNonOverlappingEnergies, single-atom trials (cbmc/interactions.cpp:54-96): overlapping trials dropped
inline std::vector<FirstBeadTrial> computeExternalNonOverlappingEnergies(const GrowContext& context,
                                                                         std::span<const rg_atom> trialPositions,
                                                                         int64_t skipBackgroundMolecule = -1)
{
  const rg_forcefield f = context.forceField().abi();
  std::vector<rg_trial_energy> out(trialPositions.size());
  check(context.ctx(),
        rg_cbmc_external_energies(context.get(), trialPositions.data(), static_cast<int>(trialPositions.size()), 1, -1,
                                  skipBackgroundMolecule, f.cutoff_framework_vdw, f.cutoff_molecule_vdw,
                                  f.cutoff_coulomb, out.data()),
        "computeExternalNonOverlappingEnergies");
  std::vector<FirstBeadTrial> energies;
  for (std::size_t i = 0; i < out.size(); ++i)
    if (!out[i].overlap) energies.push_back({trialPositions[i], fromTrial(out[i])});
  return energies;
}

// computeExternalNonOverlappingEnergies, trial sets (cbmc/interactions.cpp:98-132)
inline std::vector<ChainTrial> computeExternalNonOverlappingEnergies(const GrowContext& context,
                                                                     const std::vector<std::vector<rg_atom>>& sets,
                                                                     int skip = -1, int64_t skipBackgroundMolecule = -1)
{
  if (sets.empty()) return {};
  const std::size_t n = sets.front().size();
  std::vector<rg_atom> flat;
  for (const auto& s : sets)
  {
    if (s.size() != n) throw std::runtime_error("[raspa_b200] trial sets must have equal sizes");
    flat.insert(flat.end(), s.begin(), s.end());
  }
  const rg_forcefield f = context.forceField().abi();
  std::vector<rg_trial_energy> out(sets.size());
  check(context.ctx(),
        rg_cbmc_external_energies(context.get(), flat.data(), static_cast<int>(sets.size()), static_cast<int>(n), skip,
                                  skipBackgroundMolecule, f.cutoff_framework_vdw, f.cutoff_molecule_vdw,
                                  f.cutoff_coulomb, out.data()),
        "computeExternalNonOverlappingEnergies");
  std::vector<ChainTrial> energies;
  for (std::size_t i = 0; i < out.size(); ++i)
    if (!out[i].overlap) energies.push_back({sets[i], fromTrial(out[i])});
  return energies;
}

// computeDualCutOffCorrection (cbmc/interactions.cpp:214-251): the set with the force field's cutoffs minus with
// the dual cutoff; std::nullopt where either is dropped
inline std::optional<RunningEnergy> computeDualCutOffCorrection(const GrowContext& context,
                                                                std::span<const rg_atom> trialPositionSet,
                                                                double dualCutOff, int64_t skipBackgroundMolecule = -1)
{
  rg_trial_energy out{};
  check(context.ctx(),
        rg_cbmc_dual_cutoff_correction(context.get(), trialPositionSet.data(),
                                       static_cast<int>(trialPositionSet.size()), skipBackgroundMolecule, dualCutOff,
                                       &out),
        "computeDualCutOffCorrection");
  if (out.overlap) return std::nullopt;
  return fromTrial(out);
}
}  // namespace CBMC

namespace Interactions
{
// computeFrameworkMoleculeEnergyDifference (interactions/framework_molecule.cpp:117-252) on the framework, grids and
// force field of `context`; std::nullopt when a new atom overlaps
inline std::optional<RunningEnergy> computeFrameworkMoleculeEnergyDifference(const CBMC::GrowContext& context,
                                                                             std::span<const rg_atom> newatoms,
                                                                             std::span<const rg_atom> oldatoms)
{
  rg_trial_energy out{};
  check(context.ctx(),
        rg_framework_molecule_energy_difference(context.get(), context.forceField().chargeMethod, newatoms.data(),
                                                static_cast<int>(newatoms.size()), oldatoms.data(),
                                                static_cast<int>(oldatoms.size()), &out),
        "computeFrameworkMoleculeEnergyDifference");
  if (out.overlap) return std::nullopt;
  return CBMC::fromTrial(out);
}

// computeInterMolecularEnergyDifference (interactions/intermolecular.cpp:198-290) against the adsorbate atoms stored
// in `context`; std::nullopt when a new atom overlaps
inline std::optional<RunningEnergy> computeInterMolecularEnergyDifference(const CBMC::GrowContext& context,
                                                                          std::span<const rg_atom> newatoms,
                                                                          std::span<const rg_atom> oldatoms)
{
  rg_trial_energy out{};
  check(context.ctx(),
        rg_intermolecular_energy_difference(context.get(), newatoms.data(), static_cast<int>(newatoms.size()),
                                            oldatoms.data(), static_cast<int>(oldatoms.size()), &out),
        "computeInterMolecularEnergyDifference");
  if (out.overlap) return std::nullopt;
  return CBMC::fromTrial(out);
}
}  // namespace Interactions
}  // namespace raspa_b200

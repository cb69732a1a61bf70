// C++ parity tests through the host layer (raspa3_b200/host/raspa_b200.hpp) and the C-ABI, written the way the
// reference's own tests are (tests/raspakit-tests/ewald.cpp, tests/raspakit-tests/cbmc_interactions.cpp): the same
// systems, the same calls, the same golden values and tolerances. Needs a CUDA device.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../raspa3_b200/host/raspa_b200.hpp"

using namespace raspa_b200;

static int failures = 0;
#define EXPECT_NEAR(a, b, tol)                                                                                  \
  do                                                                                                            \
  {                                                                                                             \
    const double _a = (a), _b = (b);                                                                            \
    if (!(std::fabs(_a - _b) <= (tol)))                                                                         \
    {                                                                                                           \
      std::printf("FAILED %s:%d: %s = %.10f, expected %.10f (tol %g)\n", __FILE__, __LINE__, #a, _a, _b, (tol)); \
      ++failures;                                                                                               \
    }                                                                                                           \
  } while (0)

// units (src/raspakit/units.cpp:14-98)
static const double kPi = 3.141592653589793238462643383279502884;
static const double EnergyConversionFactor = 1.6605402e-27 * 1e-10 * 1e-10 / (1e-12 * 1e-12);
static const double EnergyToKelvin = EnergyConversionFactor * 6.0221419947e23 / 8.314464919;
static const double KelvinToEnergy = 8.314464919 / (EnergyConversionFactor * 6.0221419947e23);
static const double CoulombicConversionFactor =
    1.60217733e-19 * 1.60217733e-19 / (4.0 * kPi * 8.8541878176e-12 * 1e-10 * EnergyConversionFactor);

// Pseudo-atoms of ForceField::makeZeoliteForceField used here (forcefield.cpp:1777-1842): Si, O, CH4, C_co2, O_co2
enum Type
{
  Si = 0,
  O = 1,
  CH4 = 2,
  C_co2 = 3,
  O_co2 = 4
};

static ForceField zeoliteForceField(double rc, bool useCharge)
{
  const double eps[5] = {22.0, 53.0, 158.5, 29.933, 85.671};
  const double sig[5] = {2.30, 3.30, 3.72, 2.745, 3.017};
  const bool framework[5] = {true, true, false, false, false};
  ForceField ff;
  const int n = 5;
  ff.numberOfPseudoAtoms = n;
  ff.epsilon.resize(n * n);
  ff.sigma.resize(n * n);
  ff.shift.resize(n * n);
  ff.lj.assign(n * n, 1);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
    {
      // Lorentz-Berthelot (forcefield.cpp:924-960), shift at the cutoff (forcefield.cpp:1038-1051)
      const double e = (i == j) ? eps[i] * KelvinToEnergy
                                : std::sqrt(eps[i] * KelvinToEnergy * eps[j] * KelvinToEnergy);
      const double s = (i == j) ? sig[i] : 0.5 * (sig[i] + sig[j]);
      ff.epsilon[i * n + j] = e;
      ff.sigma[i * n + j] = s;
      const double cut = (framework[i] || framework[j]) ? rc : rc;
      const double t = (cut * cut) / (s * s);
      const double rri3 = 1.0 / (t * t * t);
      ff.shift[i * n + j] = 4.0 * e * (rri3 * (rri3 - 1.0));
    }
  ff.cutOffFrameworkVDW = ff.cutOffMoleculeVDW = ff.cutOffCoulomb = rc;
  ff.useCharge = useCharge;
  return ff;
}

// the automatic Ewald alpha that System's constructor sets (ForceField::initializeEwaldParameters,
// src/raspakit/forcefield/forcefield.cpp:1415-1424), precision 1e-6
static double automaticEwaldAlpha(double cutOffCoulomb)
{
  const double eps = 1e-6;
  const double tol = std::sqrt(std::fabs(std::log(eps * cutOffCoulomb)));
  return std::sqrt(std::fabs(std::log(eps * cutOffCoulomb * tol))) / cutOffCoulomb;
}

static rg_atom atom(double x, double y, double z, double q, int type, uint32_t mol)
{
  rg_atom a{};
  a.x = x;
  a.y = y;
  a.z = z;
  a.charge = q;
  a.scaling_vdw = 1.0;
  a.scaling_coulomb = 1.0;
  a.molecule_id = mol;
  a.type = static_cast<uint16_t>(type);
  return a;
}

// Component::makeCO2 geometry (O, C, O), C-O 1.149 Angstrom, charges of the zeolite force field
static std::vector<rg_atom> co2(double x, double y, double z, uint32_t mol)
{
  return {atom(x, y, z + 1.149, -0.3256, O_co2, mol), atom(x, y, z, 0.6512, C_co2, mol),
          atom(x, y, z - 1.149, -0.3256, O_co2, mol)};
}

// Framework::makeITQ29 (framework.cpp:1561-1590): Hall 517 (P m -3 m): all signed permutations of (x, y, z),
// fract, de-duplicated within 0.1 Angstrom (cif_reader.cpp:589-631)
static std::vector<rg_atom> itq29(int rep)
{
  const double a = 11.8671;
  struct Asym
  {
    double p[3];
    int type;
    double q;
  };
  const Asym asym[4] = {{{0.3683, 0.1847, 0.0}, Si, 2.05},
                        {{0.5, 0.2179, 0.0}, O, -1.025},
                        {{0.2939, 0.2939, 0.0}, O, -1.025},
                        {{0.3429, 0.1098, 0.1098}, O, -1.025}};
  std::vector<std::array<double, 5>> expanded;
  const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  for (const Asym& at : asym)
    for (const auto& pm : perms)
      for (int sgn = 0; sgn < 8; ++sgn)
      {
        std::array<double, 5> e{};
        for (int d = 0; d < 3; ++d)
        {
          double v = ((sgn >> d) & 1 ? -1.0 : 1.0) * at.p[pm[d]];
          v -= std::rint(v);
          if (v < 0.0) v += 1.0;
          if (v > 1.0) v -= 1.0;
          e[d] = v;
        }
        e[3] = at.type;
        e[4] = at.q;
        expanded.push_back(e);
      }
  std::vector<std::array<double, 5>> unique;
  for (std::size_t i = 0; i < expanded.size(); ++i)
  {
    bool overlap = false;
    for (std::size_t j = i + 1; j < expanded.size() && !overlap; ++j)
    {
      double r2 = 0.0;
      for (int d = 0; d < 3; ++d)
      {
        double dd = (expanded[i][d] - expanded[j][d]) * a;
        dd -= std::rint(dd / a) * a;
        r2 += dd * dd;
      }
      overlap = r2 < 0.01;
    }
    if (!overlap) unique.push_back(expanded[i]);
  }
  std::vector<rg_atom> atoms;
  for (int i = 0; i < rep; ++i)
    for (int j = 0; j < rep; ++j)
      for (int k = 0; k < rep; ++k)
        for (const auto& u : unique)
          atoms.push_back(atom((u[0] + i) * a, (u[1] + j) * a, (u[2] + k) * a, u[4], static_cast<int>(u[3]), 0));
  return atoms;
}

static rg_box cubic(double L) { return makeBox({{{L, 0, 0}, {0, L, 0}, {0, 0, L}}}); }

int main()
{
  Context ctx(0);

  {  // Ewald.Test_2_CO2_in_Box_10_10_10 (tests/raspakit-tests/ewald.cpp:25-54)
    ForceField ff = zeoliteForceField(12.0, true);
    ff.EwaldAlpha = 0.25;
    ff.numberOfWaveVectors = {8, 8, 8};
    Interactions::EwaldState ewald(ctx, ff, cubic(10.0));
    std::vector<rg_atom> atoms = co2(-1.0, 0.0, 0.0, 0);
    std::vector<rg_atom> second = co2(1.0, 0.0, 0.0, 1);
    atoms.insert(atoms.end(), second.begin(), second.end());
    const std::vector<int32_t> sizes{3, 3};
    RunningEnergy energy = Interactions::computeEwaldFourierEnergy(ewald, atoms, sizes);
    EXPECT_NEAR(energy.ewaldFourier() * EnergyToKelvin, 90.54613836, 1e-6);
  }

  for (int rep : {1, 2})
  {  // Ewald.Test_2_CO2_in_ITQ_29_1x1x1 / 2x2x2 (tests/raspakit-tests/ewald.cpp:146-210)
    ForceField ff = zeoliteForceField(12.0, true);
    ff.EwaldAlpha = 0.25;
    ff.numberOfWaveVectors = {8, 8, 8};
    const std::vector<rg_atom> fw = itq29(rep);
    Interactions::EwaldState ewald(ctx, ff, cubic(11.8671 * rep));
    Interactions::precomputeEwaldFourierRigid(ewald, fw);
    std::vector<rg_atom> atoms = co2(5.93355, 7.93355, 5.93355, 0);
    std::vector<rg_atom> second = co2(5.93355, 3.93355, 5.93355, 1);
    atoms.insert(atoms.end(), second.begin(), second.end());
    const std::vector<int32_t> sizes{3, 3};
    RunningEnergy energy = Interactions::computeEwaldFourierEnergy(ewald, atoms, sizes);
    // computeEwaldFourierEnergySingleIon of a unit charge (ewald.cpp:210-274) from the single-ion Fourier sum
    const double uIon = -(ewald.singleIonFourierSum() - CoulombicConversionFactor * 0.25 / std::sqrt(kPi));
    EXPECT_NEAR(uIon * EnergyToKelvin, rep == 1 ? 17464.2371790130 : 9673.9032373025, 1e-6);
    EXPECT_NEAR(energy.ewaldFourier() * EnergyToKelvin, rep == 1 ? -702.65863478 : -721.64644486, 1e-6);

    // energyDifferenceEwaldFourier == difference of full recomputations; acceptEwaldMove keeps it consistent
    std::vector<rg_atom> moved = co2(5.93355 + 0.37, 3.93355 - 0.21, 5.93355 + 0.5, 1);
    RunningEnergy delta = Interactions::energyDifferenceEwaldFourier(
        ewald, moved, std::span<const rg_atom>(atoms.data() + 3, 3));
    Interactions::acceptEwaldMove(ewald);
    std::vector<rg_atom> after(atoms.begin(), atoms.begin() + 3);
    after.insert(after.end(), moved.begin(), moved.end());
    RunningEnergy full = Interactions::computeEwaldFourierEnergy(ewald, after, sizes);
    EXPECT_NEAR(energy.ewaldFourier() + delta.ewaldFourier(), full.ewaldFourier(), 1e-8 * std::fabs(full.ewaldFourier()));
  }

  {  // cbmc_interactions.framework_molecule_1 / _2 (tests/raspakit-tests/cbmc_interactions.cpp:27-90)
    ForceField ff = zeoliteForceField(12.0, false);
    const std::vector<rg_atom> fw = itq29(1);
    const double a = 11.8671;
    CBMC::GrowContext context(ctx, ff, cubic(a), fw);
    const std::vector<rg_atom> one{atom(0.5 * a, 0.5 * a, 0.5 * a, 0.0, CH4, 0)};
    context.setMoleculeAtoms({});
    auto e1 = CBMC::computeExternalNonOverlappingEnergies(context, one);
    EXPECT_NEAR(e1.size(), 1.0, 0.0);
    if (!e1.empty()) EXPECT_NEAR(e1[0].energy.frameworkMoleculeVDW * EnergyToKelvin, -337.77056357, 1e-6);

    const std::vector<rg_atom> two{atom(0.5 * a, 0.5 * a, 0.5 * a, 0.0, CH4, 0),
                                   atom(0.6 * a, 0.7 * a, 0.65 * a, 0.0, CH4, 1)};
    context.setMoleculeAtoms(two);
    auto e2 = CBMC::computeExternalNonOverlappingEnergies(context, two);
    EXPECT_NEAR(e2.size(), 2.0, 0.0);
    if (e2.size() == 2)
    {
      EXPECT_NEAR((e2[0].energy.frameworkMoleculeVDW + e2[1].energy.frameworkMoleculeVDW) * EnergyToKelvin,
                  -1599.10322574, 1e-6);
      EXPECT_NEAR(e2[0].energy.moleculeMoleculeVDW * EnergyToKelvin, 2352.42793591, 1e-6);
      EXPECT_NEAR(e2[1].energy.moleculeMoleculeVDW * EnergyToKelvin, 2352.42793591, 1e-6);
    }
  }

  {  // static_energy.Test_2_CO2_in_ITQ_29_1x1x1 (tests/raspakit-tests/static_energy.cpp:21-46): the real-space Ewald
     // Coulomb pair and the Lennard-Jones pair, framework-molecule and molecule-molecule, charged framework
    ForceField ff = zeoliteForceField(12.0, true);
    ff.EwaldAlpha = automaticEwaldAlpha(12.0);
    const std::vector<rg_atom> fw = itq29(1);
    CBMC::GrowContext context(ctx, ff, cubic(11.8671), fw);
    std::vector<rg_atom> atoms = co2(5.93355, 7.93355, 5.93355, 0);
    std::vector<rg_atom> second = co2(5.93355, 3.93355, 5.93355, 1);
    atoms.insert(atoms.end(), second.begin(), second.end());
    context.setMoleculeAtoms(atoms);
    auto e = CBMC::computeExternalNonOverlappingEnergies(context, atoms);  // one trial per atom
    EXPECT_NEAR(e.size(), 6.0, 0.0);
    if (e.size() == 6)
    {
      double fwVDW = 0.0, fwCharge = 0.0, mmVDW = 0.0, mmCharge = 0.0;
      for (std::size_t i = 0; i < 6; ++i)
      {
        fwVDW += e[i].energy.frameworkMoleculeVDW;
        fwCharge += e[i].energy.frameworkMoleculeCharge;
      }
      for (std::size_t i = 0; i < 3; ++i)  // the first CO2 against the second: every intermolecular pair once
      {
        mmVDW += e[i].energy.moleculeMoleculeVDW;
        mmCharge += e[i].energy.moleculeMoleculeCharge;
      }
      EXPECT_NEAR(fwVDW * EnergyToKelvin, -1545.62921755, 1e-6);
      EXPECT_NEAR(fwCharge * EnergyToKelvin, -592.13188606, 1e-6);
      EXPECT_NEAR(mmVDW * EnergyToKelvin, -242.42459776, 1e-6);
      EXPECT_NEAR(mmCharge * EnergyToKelvin, 154.11883595, 1e-6);
    }

    // a translation of the second CO2 through the difference shims (the translation move's calls,
    // mc_moves/component/translation.cpp:30-200) equals the change of the energies above
    std::vector<rg_atom> moved = co2(5.93355 + 0.41, 3.93355 - 0.27, 5.93355 + 0.33, 1);
    std::span<const rg_atom> old(atoms.data() + 3, 3);
    auto dFramework = Interactions::computeFrameworkMoleculeEnergyDifference(context, moved, old);
    auto dMolecule = Interactions::computeInterMolecularEnergyDifference(context, moved, old);
    EXPECT_NEAR(dFramework.has_value() && dMolecule.has_value() ? 1.0 : 0.0, 1.0, 0.0);
    std::vector<rg_atom> after(atoms.begin(), atoms.begin() + 3);
    after.insert(after.end(), moved.begin(), moved.end());
    auto eNew = CBMC::computeExternalNonOverlappingEnergies(context, moved);
    auto eOld = CBMC::computeExternalNonOverlappingEnergies(context, std::vector<rg_atom>(old.begin(), old.end()));
    if (dFramework && dMolecule && eNew.size() == 3 && eOld.size() == 3)
    {
      double fv = 0.0, fq = 0.0, mv = 0.0, mq = 0.0;
      for (int i = 0; i < 3; ++i)
      {
        fv += eNew[i].energy.frameworkMoleculeVDW - eOld[i].energy.frameworkMoleculeVDW;
        fq += eNew[i].energy.frameworkMoleculeCharge - eOld[i].energy.frameworkMoleculeCharge;
        mv += eNew[i].energy.moleculeMoleculeVDW - eOld[i].energy.moleculeMoleculeVDW;
        mq += eNew[i].energy.moleculeMoleculeCharge - eOld[i].energy.moleculeMoleculeCharge;
      }
      EXPECT_NEAR(dFramework->frameworkMoleculeVDW, fv, 1e-9 * std::fabs(fv) + 1e-12);
      EXPECT_NEAR(dFramework->frameworkMoleculeCharge, fq, 1e-9 * std::fabs(fq) + 1e-12);
      EXPECT_NEAR(dMolecule->moleculeMoleculeVDW, mv, 1e-9 * std::fabs(mv) + 1e-12);
      EXPECT_NEAR(dMolecule->moleculeMoleculeCharge, mq, 1e-9 * std::fabs(mq) + 1e-12);
    }
    // accepted: the stored atoms follow, and moving back gives the opposite difference
    context.updateMoleculeAtoms(3, moved);
    auto back = Interactions::computeInterMolecularEnergyDifference(context, old, moved);
    if (back && dMolecule)
      EXPECT_NEAR(back->moleculeMoleculeCharge, -dMolecule->moleculeMoleculeCharge,
                  1e-9 * std::fabs(dMolecule->moleculeMoleculeCharge) + 1e-12);
  }

  {  // grid build through InterpolationEnergyGrid, then the grid branch of the trial energies
    ForceField ff = zeoliteForceField(12.0, false);
    const std::vector<rg_atom> fw = itq29(1);
    const double a = 11.8671;
    InterpolationEnergyGrid grid(cubic(a), {48, 48, 48});
    grid.makeFrameworkInterpolationGrid(ctx, InterpolationGridType::LennardJones, ff, fw, 12.0, CH4);
    CBMC::GrowContext context(ctx, ff, cubic(a), fw);
    context.setInterpolationGrid(CH4, grid);
    context.setMoleculeAtoms({});
    const std::vector<rg_atom> one{atom(0.5 * a, 0.5 * a, 0.5 * a, 0.0, CH4, 0)};
    auto e = CBMC::computeExternalNonOverlappingEnergies(context, one);
    // The grid holds the sum over every periodic image within the cutoff. In the 11.87 A cell the minimum-image pair
    // loop (and the -337.77 K golden) misses the images beyond half a cell, so the exact value is the pair loop in the
    // 3x3x3 supercell, where the minimum image reaches all of them. Tolerance: interpolation error at 0.25 A spacing.
    CBMC::GrowContext exact(ctx, ff, cubic(3.0 * a), itq29(3));
    exact.setMoleculeAtoms({});
    auto ex = CBMC::computeExternalNonOverlappingEnergies(exact, one);
    EXPECT_NEAR(ex.size(), 1.0, 0.0);
    if (!e.empty() && !ex.empty())
      EXPECT_NEAR(e[0].energy.frameworkMoleculeVDW, ex[0].energy.frameworkMoleculeVDW,
                  1e-3 * std::fabs(ex[0].energy.frameworkMoleculeVDW));
  }

  {  // the triquintic scheme through the same class: at the grid points its energy channel is the same pair sum as
     // the tricubic grid's, and its first-derivative channels equal the tricubic ones (away from overlap-clamped
     // points, whose derivative channels are the rounding residue of cancelling terms of ~1e10)
    ForceField ff = zeoliteForceField(12.0, false);
    const std::vector<rg_atom> fw = itq29(1);
    const double a = 11.8671;
    InterpolationEnergyGrid cubicGrid(cubic(a), {12, 12, 12});
    InterpolationEnergyGrid quinticGrid(cubic(a), {12, 12, 12}, InterpolationScheme::Triquintic);
    cubicGrid.makeFrameworkInterpolationGrid(ctx, InterpolationGridType::LennardJones, ff, fw, 12.0, CH4);
    quinticGrid.makeFrameworkInterpolationGrid(ctx, InterpolationGridType::LennardJones, ff, fw, 12.0, CH4);
    EXPECT_NEAR(static_cast<double>(quinticGrid.data.size()), 27.0 * 12 * 12 * 12, 0.0);
    double worst = 0.0;
    for (std::size_t pt = 0; pt < 12 * 12 * 12; ++pt)
      for (int l = 0; l < 4; ++l)
      {
        if (cubicGrid.data[8 * pt] >= 2.0 * ff.energyOverlapCriteria) continue;
        const double c = cubicGrid.data[8 * pt + l], q = quinticGrid.data[27 * pt + l];
        worst = std::fmax(worst, std::fabs(c - q) / std::fmax(1.0, std::fabs(c)));
      }
    EXPECT_NEAR(worst, 0.0, 1e-8);  // FP64 sums of terms up to ~1e6 near the overlap region (3.3e-9 measured)
  }

  std::printf("%s (%d failures)\n", failures ? "FAILED" : "PASSED", failures);
  return failures ? 1 : 0;
}

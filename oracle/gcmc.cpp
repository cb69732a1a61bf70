// FP64 CPU GCMC of rigid molecules with interpolation grids and Ewald summation — TEST INFRASTRUCTURE ONLY.
//
// Restates the reference's Monte Carlo moves for one rigid component in a rigid framework:
//   translation   mc_moves/component/translation.cpp:30-200 (one random Cartesian direction, uniform in +-max)
//   rotation      mc_moves/component/rotation.cpp:30-190 (one random Cartesian axis, angle uniform in +-max, about the
//                 centre of mass)
//   CBMC insertion mc_moves/component/insertion_cbmc.cpp:34-207 with cbmc/multiple_first_bead.cpp:20-49 (k uniform
//                 first-bead positions) and the rigid seed step of cbmc/operators.cpp:951-970 (k uniform orientations
//                 about the first bead), Pacc = exp(-beta dU_ewald) beta f V / (N+1) W / W_IG with W_IG = 1
//   CBMC deletion mc_moves/component/deletion_cbmc.cpp:34-195 with cbmc/multiple_first_bead.cpp:51-76 (trial 0 = the
//                 old position / orientation), Pacc = exp(-beta dU_ewald) N / (beta f V) W_IG / W
// Framework-molecule energies use the tricubic grids (cbmc/interactions_framework_molecule.cpp:57-69), molecule-
// molecule energies the Lennard-Jones and real-space Ewald pair sums (cbmc/interactions_intermolecular.cpp:22-95),
// and the Fourier part energyDifferenceEwaldFourier (interactions/ewald.cpp:1043-1244) on stored structure factors
// that include the framework. Independent chains run in parallel (OpenMP), one chain per thread.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "rng.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
constexpr double kPi = 3.141592653589793238462643383279502884;

using oracle_rng::Rng;

void randomRotation(Rng& r, double R[3][3])
{
  // uniform unit quaternion (Shoemake) -> rotation matrix
  const double u1 = r.uniform(), u2 = r.uniform(), u3 = r.uniform();
  const double x = std::sqrt(1 - u1) * std::sin(2 * kPi * u2), y = std::sqrt(1 - u1) * std::cos(2 * kPi * u2);
  const double z = std::sqrt(u1) * std::sin(2 * kPi * u3), w = std::sqrt(u1) * std::cos(2 * kPi * u3);
  R[0][0] = 1 - 2 * (y * y + z * z);
  R[0][1] = 2 * (x * y - z * w);
  R[0][2] = 2 * (x * z + y * w);
  R[1][0] = 2 * (x * y + z * w);
  R[1][1] = 1 - 2 * (x * x + z * z);
  R[1][2] = 2 * (y * z - x * w);
  R[2][0] = 2 * (x * z - y * w);
  R[2][1] = 2 * (y * z + x * w);
  R[2][2] = 1 - 2 * (x * x + y * y);
}

void axisRotation(int axis, double angle, double R[3][3])
{
  const double c = std::cos(angle), s = std::sin(angle);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = (i == j) ? 1.0 : 0.0;
  const int a = (axis + 1) % 3, b = (axis + 2) % 3;
  R[a][a] = c;
  R[a][b] = -s;
  R[b][a] = s;
  R[b][b] = c;
}

struct Chain
{
  const ogcmc_setup* p;
  Rng rng;
  std::vector<oatom> atoms;  // molecules consecutive, p->n_atoms each
  std::vector<double> stored;
  int n = 0;
  double energy = 0.0;
  obox box;
  double cell[3][3];  // rows = lattice vectors (box.cell[3c+r] = cell[c][r])
  double volume;
  Chain(const ogcmc_setup* setup, uint64_t seed) : p(setup), rng(seed)
  {
    box = setup->box;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) cell[c][r] = box.cell[3 * c + r];
    volume = cell[0][0] * (cell[1][1] * cell[2][2] - cell[1][2] * cell[2][1]) -
             cell[1][0] * (cell[0][1] * cell[2][2] - cell[0][2] * cell[2][1]) +
             cell[2][0] * (cell[0][1] * cell[1][2] - cell[0][2] * cell[1][1]);
  }

  void randomPosition(double out[3])
  {
    // SimulationBox::randomPosition (simulationbox.cpp:132-135): cell * (u, u, u)
    const double s0 = rng.uniform(), s1 = rng.uniform(), s2 = rng.uniform();
    for (int r = 0; r < 3; ++r) out[r] = cell[0][r] * s0 + cell[1][r] * s1 + cell[2][r] * s2;
  }

  // External energy (framework via grids + other molecules) of `set` atoms; returns false on overlap.
  bool external(const oatom* set, int count, int64_t skip_molecule, double& e)
  {
    oenergy ef, em;
    const int okf = oracle_cbmc_framework_molecule(p->ff, &box, p->grids, p->gnx, p->gny, p->gnz, &p->grid_cell,
                                                   nullptr, 0, p->ff->cutoff_framework_vdw, p->ff->cutoff_coulomb, set,
                                                   count, -1, &ef);
    if (!okf) return false;
    const int okm = oracle_cbmc_intermolecular(p->ff, &box, atoms.data(), n * p->n_atoms, p->ff->cutoff_molecule_vdw,
                                               p->ff->cutoff_coulomb, set, count, -1, skip_molecule, &em);
    if (!okm) return false;
    e = ef.framework_molecule_vdw + ef.framework_molecule_charge + em.molecule_molecule_vdw +
        em.molecule_molecule_charge;
    return true;
  }

  double ewaldDelta(const oatom* nw, int nn, const oatom* old, int no, std::vector<double>& trial)
  {
    if (!p->use_ewald) return 0.0;
    oenergy e;
    trial.resize(stored.size());
    oracle_ewald_delta(p->ff, &box, stored.data(), nw, nn, old, no, 0.0, nullptr, trial.data(), &e);
    return e.ewald_fourier + e.ewald_self + e.ewald_exclusion;
  }

  void placeMolecule(const double center[3], const double R[3][3], uint32_t mol, oatom* out)
  {
    for (int i = 0; i < p->n_atoms; ++i)
    {
      oatom a{};
      double d[3];
      for (int r = 0; r < 3; ++r)
        d[r] = R[r][0] * p->offsets[3 * i] + R[r][1] * p->offsets[3 * i + 1] + R[r][2] * p->offsets[3 * i + 2];
      a.x = center[0] + d[0];
      a.y = center[1] + d[1];
      a.z = center[2] + d[2];
      a.charge = p->charges[i];
      a.scaling_vdw = 1.0;
      a.scaling_coulomb = 1.0;
      a.molecule_id = mol;
      a.type = static_cast<uint16_t>(p->types[i]);
      out[i] = a;
    }
  }

  void centerOf(const oatom* m, double c[3])
  {
    // centre of mass (the rotation centre): the body offsets are relative to it, so it is the mass-weighted mean
    double w = 0.0;
    c[0] = c[1] = c[2] = 0.0;
    for (int i = 0; i < p->n_atoms; ++i)
    {
      c[0] += p->masses[i] * m[i].x;
      c[1] += p->masses[i] * m[i].y;
      c[2] += p->masses[i] * m[i].z;
      w += p->masses[i];
    }
    for (int d = 0; d < 3; ++d) c[d] /= w;
  }

  void relabel()
  {
    for (int m = 0; m < n; ++m)
      for (int i = 0; i < p->n_atoms; ++i) atoms[m * p->n_atoms + i].molecule_id = static_cast<uint32_t>(m);
  }

  int translateOrRotate(bool rotate)
  {
    if (n == 0) return 0;
    const int na = p->n_atoms;
    const int m = std::min(n - 1, static_cast<int>(rng.uniform() * n));
    oatom* old = &atoms[m * na];
    std::vector<oatom> nw(old, old + na);
    const int dir = std::min(2, static_cast<int>(3.0 * rng.uniform()));
    if (!rotate)
    {
      const double disp = p->max_translation * 2.0 * (rng.uniform() - 0.5);
      for (auto& a : nw) (&a.x)[dir] += disp;
    }
    else
    {
      const double angle = p->max_rotation * 2.0 * (rng.uniform() - 0.5);
      double R[3][3], c[3];
      axisRotation(dir, angle, R);
      centerOf(old, c);
      for (int i = 0; i < na; ++i)
      {
        double d[3] = {old[i].x - c[0], old[i].y - c[1], old[i].z - c[2]};
        nw[i].x = c[0] + R[0][0] * d[0] + R[0][1] * d[1] + R[0][2] * d[2];
        nw[i].y = c[1] + R[1][0] * d[0] + R[1][1] * d[1] + R[1][2] * d[2];
        nw[i].z = c[2] + R[2][0] * d[0] + R[2][1] * d[1] + R[2][2] * d[2];
      }
    }
    double eNew, eOld = 0.0;
    if (!external(nw.data(), na, m, eNew)) return 0;
    external(old, na, m, eOld);
    std::vector<double> trial;
    const double dEw = ewaldDelta(nw.data(), na, old, na, trial);
    const double dU = eNew - eOld + dEw;
    if (rng.uniform() < std::exp(-p->beta * dU))
    {
      std::copy(nw.begin(), nw.end(), old);
      if (p->use_ewald) stored.swap(trial);
      energy += dU;
      return 1;
    }
    return 0;
  }

  // CBMC first bead + rigid orientations; retrace keeps trial 0 at the existing molecule m
  bool grow(int m_retrace, std::vector<oatom>& mol, double& W, double& eExt)
  {
    const int na = p->n_atoms, sb = p->starting_bead, k1 = p->n_first_bead_trials, k2 = p->n_orientation_trials;
    const bool retrace = m_retrace >= 0;
    const uint32_t mid = retrace ? static_cast<uint32_t>(m_retrace) : static_cast<uint32_t>(n);
    const int64_t skip = retrace ? m_retrace : -1;
    oatom bead{};
    bead.charge = p->charges[sb];
    bead.scaling_vdw = bead.scaling_coulomb = 1.0;
    bead.molecule_id = mid;
    bead.type = static_cast<uint16_t>(p->types[sb]);
    std::vector<oatom> beads(k1, bead);
    for (int t = 0; t < k1; ++t)
    {
      if (retrace && t == 0)
      {
        beads[0] = atoms[m_retrace * na + sb];
        continue;
      }
      double r[3];
      randomPosition(r);
      beads[t].x = r[0];
      beads[t].y = r[1];
      beads[t].z = r[2];
    }
    std::vector<double> logBF, energies;
    std::vector<int> index;
    for (int t = 0; t < k1; ++t)
    {
      double e;
      if (!external(&beads[t], 1, skip, e)) continue;
      logBF.push_back(-p->beta * e);
      energies.push_back(e);
      index.push_back(t);
    }
    if (logBF.empty()) return false;
    int sel = retrace ? 0 : oracle_select_trial(logBF.data(), static_cast<int>(logBF.size()), rng.uniform());
    double W1 = 0.0;
    for (double x : logBF) W1 += std::exp(x);
    W1 /= static_cast<double>(k1);
    if (retrace && index[0] != 0) return false;  // the existing first bead always has a finite energy
    const oatom first = beads[index[sel]];
    const double eFirst = energies[sel];
    // orientations about the first bead
    double off0[3] = {p->offsets[3 * sb], p->offsets[3 * sb + 1], p->offsets[3 * sb + 2]};
    std::vector<std::vector<oatom>> sets(k2);
    for (int t = 0; t < k2; ++t)
    {
      if (retrace && t == 0)
      {
        sets[0].assign(atoms.begin() + m_retrace * na, atoms.begin() + (m_retrace + 1) * na);
        continue;
      }
      double R[3][3];
      randomRotation(rng, R);
      double rc[3];
      for (int r = 0; r < 3; ++r) rc[r] = R[r][0] * off0[0] + R[r][1] * off0[1] + R[r][2] * off0[2];
      double center[3] = {first.x - rc[0], first.y - rc[1], first.z - rc[2]};
      sets[t].resize(na);
      placeMolecule(center, R, mid, sets[t].data());
    }
    std::vector<double> logBF2, energies2;
    std::vector<int> index2;
    std::vector<oatom> others(na - 1);
    for (int t = 0; t < k2; ++t)
    {
      int j = 0;
      for (int i = 0; i < na; ++i)
        if (i != sb) others[j++] = sets[t][i];
      double e = 0.0;
      if (na > 1 && !external(others.data(), na - 1, skip, e)) continue;
      logBF2.push_back(-p->beta * e);
      energies2.push_back(e);
      index2.push_back(t);
    }
    if (logBF2.empty()) return false;
    int sel2 = retrace ? 0 : oracle_select_trial(logBF2.data(), static_cast<int>(logBF2.size()), rng.uniform());
    if (retrace && index2[0] != 0) return false;
    double W2 = 0.0;
    for (double x : logBF2) W2 += std::exp(x);
    W2 /= static_cast<double>(k2);
    mol = sets[index2[sel2]];
    W = W1 * W2;
    eExt = eFirst + energies2[sel2];
    return true;
  }

  int insertion()
  {
    if (n >= p->max_molecules) return 0;
    std::vector<oatom> mol;
    double W, eExt;
    if (!grow(-1, mol, W, eExt)) return 0;
    if (W < 1e-150) return 0;  // minimumRosenbluthFactor (forcefield.ixx)
    std::vector<double> trial;
    const double dEw = ewaldDelta(mol.data(), p->n_atoms, nullptr, 0, trial);
    const double pacc = std::exp(-p->beta * dEw) * p->beta * p->fugacity * volume / static_cast<double>(n + 1) * W;
    if (rng.uniform() < pacc)
    {
      atoms.insert(atoms.end(), mol.begin(), mol.end());
      ++n;
      if (p->use_ewald) stored.swap(trial);
      energy += eExt + dEw;
      return 1;
    }
    return 0;
  }

  int deletion()
  {
    if (n == 0) return 0;
    const int na = p->n_atoms;
    const int m = std::min(n - 1, static_cast<int>(rng.uniform() * n));
    std::vector<oatom> mol;
    double W, eExt;
    if (!grow(m, mol, W, eExt)) return 0;
    std::vector<double> trial;
    const double dEw = ewaldDelta(nullptr, 0, &atoms[m * na], na, trial);
    const double pacc = std::exp(-p->beta * dEw) * static_cast<double>(n) / (p->beta * p->fugacity * volume) / W;
    if (rng.uniform() < pacc)
    {
      // move the last molecule into slot m and relabel the molecule ids
      if (m != n - 1) std::copy(atoms.begin() + (n - 1) * na, atoms.begin() + n * na, atoms.begin() + m * na);
      atoms.resize((n - 1) * na);
      --n;
      relabel();
      if (p->use_ewald) stored.swap(trial);
      energy += -eExt + dEw;
      return 1;
    }
    return 0;
  }

  double recompute()
  {
    // total energy from scratch: framework (grids) + molecule-molecule (each pair once) + Ewald
    double e = 0.0;
    const int na = p->n_atoms;
    for (int m = 0; m < n; ++m)
    {
      oenergy ef;
      oracle_cbmc_framework_molecule(p->ff, &box, p->grids, p->gnx, p->gny, p->gnz, &p->grid_cell, nullptr, 0,
                                     p->ff->cutoff_framework_vdw, p->ff->cutoff_coulomb, &atoms[m * na], na, -1, &ef);
      e += ef.framework_molecule_vdw + ef.framework_molecule_charge;
      if (m + 1 < n)
      {
        oenergy em;
        oracle_cbmc_intermolecular(p->ff, &box, &atoms[(m + 1) * na], (n - m - 1) * na, p->ff->cutoff_molecule_vdw,
                                   p->ff->cutoff_coulomb, &atoms[m * na], na, -1, -1, &em);
        e += em.molecule_molecule_vdw + em.molecule_molecule_charge;
      }
    }
    if (p->use_ewald && n > 0)
    {
      std::vector<int32_t> sizes(n, na);
      oenergy ee;
      oracle_ewald_fourier_energy(p->ff, &box, p->s_framework, atoms.data(), n * na, sizes.data(), n, 0.0, nullptr,
                                  &ee);
      e += ee.ewald_fourier + ee.ewald_self + ee.ewald_exclusion;
    }
    return e;
  }
};
}  // namespace

extern "C" void oracle_gcmc_run(const ogcmc_setup* setup, int n_chains, int64_t steps, int64_t equilibration,
                                uint64_t seed, int threads, ogcmc_result* out, double* seconds)
{
  const int64_t nk = setup->use_ewald ? oracle_ewald_kvectors(setup->ff, &setup->box, nullptr, nullptr, nullptr) : 0;
  auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
  for (int c = 0; c < n_chains; ++c)
  {
    Chain ch(setup, seed * 0x100000001b3ULL + static_cast<uint64_t>(c) * 0x9e3779b97f4a7c15ULL + 1);
    ch.stored.assign(10 * nk, 0.0);
    for (int64_t k = 0; k < nk; ++k)
    {
      ch.stored[10 * k] = setup->s_framework ? setup->s_framework[2 * k] : 0.0;
      ch.stored[10 * k + 1] = setup->s_framework ? setup->s_framework[2 * k + 1] : 0.0;
    }
    ogcmc_result& r = out[c];
    std::memset(&r, 0, sizeof(r));
    const double ptot = setup->p_translation + setup->p_rotation + setup->p_swap;
    const int64_t block = steps / 5 > 0 ? steps / 5 : 1;
    double block_sum = 0.0;
    int64_t block_cnt = 0;
    int bi = 0;
    for (int64_t s = 0; s < equilibration + steps; ++s)
    {
      const double u = ch.rng.uniform() * ptot;
      int kind, acc;
      if (u < setup->p_translation)
      {
        kind = 0;
        acc = ch.translateOrRotate(false);
      }
      else if (u < setup->p_translation + setup->p_rotation)
      {
        kind = 1;
        acc = ch.translateOrRotate(true);
      }
      else if (ch.rng.uniform() < 0.5)
      {
        kind = 2;
        acc = ch.insertion();
      }
      else
      {
        kind = 3;
        acc = ch.deletion();
      }
      if (s >= equilibration)
      {
        r.attempted[kind] += 1;
        r.accepted[kind] += acc;
        r.sum_n += ch.n;
        r.sum_n2 += static_cast<double>(ch.n) * ch.n;
        r.sum_energy += ch.energy;
        r.samples += 1;
        block_sum += ch.n;
        if (++block_cnt == block && bi < 5)
        {
          r.block_n[bi++] = block_sum / static_cast<double>(block_cnt);
          block_sum = 0.0;
          block_cnt = 0;
        }
      }
    }
    r.n_molecules = ch.n;
    r.running_energy = ch.energy;
    r.recomputed_energy = ch.recompute();
  }
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
}

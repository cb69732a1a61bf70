// FP64 CPU GCMC of a mixture of rigid molecules with identity change — TEST INFRASTRUCTURE ONLY.
//
// One system, several rigid components. Moves (each picks a component uniformly, then a move by its probability):
//   translation      mc_moves/component/translation.cpp:30-200 (one Cartesian direction, uniform in +-max)
//   rotation         mc_moves/component/rotation.cpp:30-190 (one Cartesian axis about the centre of mass)
//   CBMC insertion   mc_moves/component/insertion_cbmc.cpp:34-207, first bead cbmc/multiple_first_bead.cpp:20-49,
//                    rigid orientations about it (cbmc/operators.cpp:951-970)
//   CBMC deletion    mc_moves/component/deletion_cbmc.cpp:34-195 (retrace: trial 0 is the old molecule)
//   identity change  mc_moves/component/identity_change.cpp:33-290: the new component is grown with its first bead on
//                    the old molecule's starting bead (growMultipleFirstBeadPartialInsertion,
//                    cbmc/multiple_first_bead.cpp:136-153: W = exp(-beta U) of that one bead, with the old molecule
//                    excluded from the environment), the old molecule is retraced (retraceMultipleFirstBeadPartialDeletion,
//                    :155-168), Pacc = exp(-beta dU_ewald) (W_new / W_IG_new) f_new N_old / ((W_old / W_IG_old) f_old
//                    (N_new + 1)), and old and new components are swapped with probability 1/2 first
// Framework-molecule energies from the tricubic grids, molecule-molecule pair sums (Lennard-Jones + real-space Ewald),
// and the Ewald Fourier difference on stored structure factors that include the framework.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "rng.h"

namespace
{
using oracle_rng::Rng;
constexpr double kPi = 3.141592653589793238462643383279502884;

void randomRotation(Rng& r, double R[3][3])
{
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

struct Mixture
{
  const omix_setup* p;
  Rng rng;
  int na;                   // atoms per molecule (the same for every component)
  std::vector<oatom> atoms;  // molecules consecutive, na atoms each
  std::vector<int> comp;     // component of each molecule
  std::vector<double> stored;
  int n = 0;
  int count[4] = {0, 0, 0, 0};
  double energy = 0.0;
  double cell[3][3];
  double volume;

  Mixture(const omix_setup* setup, uint64_t seed) : p(setup), rng(seed), na(setup->comps[0].n_atoms)
  {
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) cell[c][r] = p->box.cell[3 * c + r];
    volume = cell[0][0] * (cell[1][1] * cell[2][2] - cell[1][2] * cell[2][1]) -
             cell[1][0] * (cell[0][1] * cell[2][2] - cell[0][2] * cell[2][1]) +
             cell[2][0] * (cell[0][1] * cell[1][2] - cell[0][2] * cell[1][1]);
  }

  void randomPosition(double out[3])
  {
    const double s0 = rng.uniform(), s1 = rng.uniform(), s2 = rng.uniform();
    for (int r = 0; r < 3; ++r) out[r] = cell[0][r] * s0 + cell[1][r] * s1 + cell[2][r] * s2;
  }

  // framework (grids) + molecule-molecule energy of `count` atoms, excluding molecule `skip`; false on overlap
  bool external(const oatom* set, int cnt, int64_t skip, double& e)
  {
    oenergy ef, em;
    if (!oracle_cbmc_framework_molecule(p->ff, &p->box, p->grids, p->gnx, p->gny, p->gnz, &p->grid_cell, p->framework,
                                        p->n_framework,
                                        p->ff->cutoff_framework_vdw, p->ff->cutoff_coulomb, set, cnt, -1, &ef))
      return false;
    if (!oracle_cbmc_intermolecular(p->ff, &p->box, atoms.data(), n * na, p->ff->cutoff_molecule_vdw,
                                    p->ff->cutoff_coulomb, set, cnt, -1, skip, &em))
      return false;
    e = ef.framework_molecule_vdw + ef.framework_molecule_charge + em.molecule_molecule_vdw +
        em.molecule_molecule_charge;
    return true;
  }

  double ewaldDelta(const oatom* nw, int nn, const oatom* old, int no, std::vector<double>& trial)
  {
    if (!p->use_ewald) return 0.0;
    oenergy e;
    trial.resize(stored.size());
    oracle_ewald_delta(p->ff, &p->box, stored.data(), nw, nn, old, no, 0.0, nullptr, trial.data(), &e);
    return e.ewald_fourier + e.ewald_self + e.ewald_exclusion;
  }

  void place(const omix_component& c, const double center[3], const double R[3][3], uint32_t mol, oatom* out)
  {
    for (int i = 0; i < c.n_atoms; ++i)
    {
      oatom a{};
      double d[3];
      for (int r = 0; r < 3; ++r)
        d[r] = R[r][0] * c.offsets[3 * i] + R[r][1] * c.offsets[3 * i + 1] + R[r][2] * c.offsets[3 * i + 2];
      a.x = center[0] + d[0];
      a.y = center[1] + d[1];
      a.z = center[2] + d[2];
      a.charge = c.charges[i];
      a.scaling_vdw = a.scaling_coulomb = 1.0;
      a.molecule_id = mol;
      a.type = static_cast<uint16_t>(c.types[i]);
      out[i] = a;
    }
  }

  void centerOf(const omix_component& c, const oatom* m, double out[3])
  {
    double w = 0.0;
    out[0] = out[1] = out[2] = 0.0;
    for (int i = 0; i < c.n_atoms; ++i)
    {
      out[0] += c.masses[i] * m[i].x;
      out[1] += c.masses[i] * m[i].y;
      out[2] += c.masses[i] * m[i].z;
      w += c.masses[i];
    }
    for (int d = 0; d < 3; ++d) out[d] /= w;
  }

  void relabel()
  {
    for (int m = 0; m < n; ++m)
      for (int i = 0; i < na; ++i) atoms[m * na + i].molecule_id = static_cast<uint32_t>(m);
  }

  // the k-th molecule of component c (k < count[c])
  int nthOf(int c, int k)
  {
    for (int m = 0; m < n; ++m)
      if (comp[m] == c && k-- == 0) return m;
    return -1;
  }

  int translateOrRotate(int c, bool rotate)
  {
    if (count[c] == 0) return 0;
    const int m = nthOf(c, std::min(count[c] - 1, static_cast<int>(rng.uniform() * count[c])));
    const omix_component& cc = p->comps[c];
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
      const double cs = std::cos(angle), sn = std::sin(angle);
      const int a1 = (dir + 1) % 3, a2 = (dir + 2) % 3;
      double ctr[3];
      centerOf(cc, old, ctr);
      for (int i = 0; i < na; ++i)
      {
        double d[3] = {old[i].x - ctr[0], old[i].y - ctr[1], old[i].z - ctr[2]};
        double r[3] = {d[0], d[1], d[2]};
        r[a1] = cs * d[a1] - sn * d[a2];
        r[a2] = sn * d[a1] + cs * d[a2];
        nw[i].x = ctr[0] + r[0];
        nw[i].y = ctr[1] + r[1];
        nw[i].z = ctr[2] + r[2];
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

  // Rigid CBMC growth of component c. mode 0: insertion (k1 uniform first beads); mode 1: retrace of molecule m
  // (trial 0 = old); mode 2: identity-change growth with the first bead fixed at `fixed` and molecule `skip` excluded;
  // mode 3: identity-change retrace of molecule m (first bead fixed at its own position).
  bool grow(int c, int mode, int m, const double* fixed, int64_t skip, std::vector<oatom>& mol, double& W, double& eExt)
  {
    const omix_component& cc = p->comps[c];
    const int sb = cc.starting_bead;
    const bool retrace = mode == 1 || mode == 3;
    const int k1 = (mode >= 2) ? 1 : p->n_first_bead_trials, k2 = p->n_orientation_trials;
    const uint32_t mid = retrace ? static_cast<uint32_t>(m) : static_cast<uint32_t>(n);
    oatom bead{};
    bead.charge = cc.charges[sb];
    bead.scaling_vdw = bead.scaling_coulomb = 1.0;
    bead.molecule_id = mid;
    bead.type = static_cast<uint16_t>(cc.types[sb]);
    std::vector<oatom> beads(k1, bead);
    for (int t = 0; t < k1; ++t)
    {
      if (retrace && t == 0)
      {
        beads[0] = atoms[m * na + sb];
        continue;
      }
      double r[3];
      if (mode == 2)
        std::copy(fixed, fixed + 3, r);
      else
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
      if (!external(&beads[t], 1, retrace ? m : skip, e)) continue;
      logBF.push_back(-p->beta * e);
      energies.push_back(e);
      index.push_back(t);
    }
    if (logBF.empty()) return false;
    if (retrace && index[0] != 0) return false;
    int sel = 0;
    double W1 = 0.0;
    if (mode >= 2)
      W1 = std::exp(logBF[0]);  // partial insertion / deletion: one fixed bead, no division by k
    else
    {
      sel = retrace ? 0 : oracle_select_trial(logBF.data(), static_cast<int>(logBF.size()), rng.uniform());
      for (double x : logBF) W1 += std::exp(x);
      W1 /= static_cast<double>(k1);
    }
    const oatom first = beads[index[sel]];
    const double eFirst = energies[sel];
    const double off0[3] = {cc.offsets[3 * sb], cc.offsets[3 * sb + 1], cc.offsets[3 * sb + 2]};
    std::vector<std::vector<oatom>> sets(k2);
    for (int t = 0; t < k2; ++t)
    {
      if (retrace && t == 0)
      {
        sets[0].assign(atoms.begin() + m * na, atoms.begin() + (m + 1) * na);
        continue;
      }
      double R[3][3];
      randomRotation(rng, R);
      double rc[3];
      for (int r = 0; r < 3; ++r) rc[r] = R[r][0] * off0[0] + R[r][1] * off0[1] + R[r][2] * off0[2];
      const double center[3] = {first.x - rc[0], first.y - rc[1], first.z - rc[2]};
      sets[t].resize(na);
      place(cc, center, R, mid, sets[t].data());
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
      if (na > 1 && !external(others.data(), na - 1, retrace ? m : skip, e)) continue;
      logBF2.push_back(-p->beta * e);
      energies2.push_back(e);
      index2.push_back(t);
    }
    if (logBF2.empty()) return false;
    if (retrace && index2[0] != 0) return false;
    const int sel2 = retrace ? 0 : oracle_select_trial(logBF2.data(), static_cast<int>(logBF2.size()), rng.uniform());
    double W2 = 0.0;
    for (double x : logBF2) W2 += std::exp(x);
    W2 /= static_cast<double>(k2);
    mol = sets[index2[sel2]];
    W = W1 * W2;
    eExt = eFirst + energies2[sel2];
    return true;
  }

  int insertion(int c)
  {
    if (n >= p->max_molecules) return 0;
    std::vector<oatom> mol;
    double W, eExt;
    if (!grow(c, 0, -1, nullptr, -1, mol, W, eExt)) return 0;
    if (W < 1e-150) return 0;
    std::vector<double> trial;
    const double dEw = ewaldDelta(mol.data(), na, nullptr, 0, trial);
    const omix_component& cc = p->comps[c];
    const double pacc = std::exp(-p->beta * dEw) * p->beta * cc.fugacity * volume /
                        static_cast<double>(count[c] + 1) * W / cc.w_ig;
    if (rng.uniform() < pacc)
    {
      atoms.insert(atoms.end(), mol.begin(), mol.end());
      comp.push_back(c);
      ++n;
      ++count[c];
      if (p->use_ewald) stored.swap(trial);
      energy += eExt + dEw;
      return 1;
    }
    return 0;
  }

  void remove(int m)
  {
    const int c = comp[m];
    if (m != n - 1)
    {
      std::copy(atoms.begin() + (n - 1) * na, atoms.begin() + n * na, atoms.begin() + m * na);
      comp[m] = comp[n - 1];
    }
    atoms.resize((n - 1) * na);
    comp.pop_back();
    --n;
    --count[c];
    relabel();
  }

  int deletion(int c)
  {
    if (count[c] == 0) return 0;
    const int m = nthOf(c, std::min(count[c] - 1, static_cast<int>(rng.uniform() * count[c])));
    std::vector<oatom> mol;
    double W, eExt;
    if (!grow(c, 1, m, nullptr, -1, mol, W, eExt)) return 0;
    std::vector<double> trial;
    const double dEw = ewaldDelta(nullptr, 0, &atoms[m * na], na, trial);
    const omix_component& cc = p->comps[c];
    const double pacc = std::exp(-p->beta * dEw) * static_cast<double>(count[c]) / (p->beta * cc.fugacity * volume) *
                        cc.w_ig / W;
    if (rng.uniform() < pacc)
    {
      remove(m);
      if (p->use_ewald) stored.swap(trial);
      energy += -eExt + dEw;
      return 1;
    }
    return 0;
  }

  int identityChange(int c)
  {
    if (p->n_components < 2) return 0;
    int oldC = c, newC = (c + 1 + static_cast<int>(rng.uniform() * (p->n_components - 1))) % p->n_components;
    if (rng.uniform() < 0.5) std::swap(oldC, newC);
    if (count[oldC] == 0) return 0;
    const int m = nthOf(oldC, std::min(count[oldC] - 1, static_cast<int>(rng.uniform() * count[oldC])));
    const omix_component& co = p->comps[oldC];
    const omix_component& cn = p->comps[newC];
    const oatom& sbOld = atoms[m * na + co.starting_bead];
    const double fixed[3] = {sbOld.x, sbOld.y, sbOld.z};
    std::vector<oatom> mol, dummy;
    double Wn, eN, Wo, eO;
    if (!grow(newC, 2, -1, fixed, m, mol, Wn, eN)) return 0;
    if (Wn < 1e-150) return 0;
    if (!grow(oldC, 3, m, nullptr, -1, dummy, Wo, eO)) return 0;
    std::vector<double> trial;
    const double dEw = ewaldDelta(mol.data(), na, &atoms[m * na], na, trial);
    const double pacc = std::exp(-p->beta * dEw) * (Wn / cn.w_ig) * cn.fugacity * static_cast<double>(count[oldC]) /
                        ((Wo / co.w_ig) * co.fugacity * static_cast<double>(count[newC] + 1));
    if (rng.uniform() < pacc)
    {
      // the new molecule takes the old one's slot
      for (int i = 0; i < na; ++i)
      {
        mol[i].molecule_id = static_cast<uint32_t>(m);
        atoms[m * na + i] = mol[i];
      }
      comp[m] = newC;
      --count[oldC];
      ++count[newC];
      if (p->use_ewald) stored.swap(trial);
      energy += (eN - eO) + dEw;
      return 1;
    }
    return 0;
  }

  double recompute()
  {
    double e = 0.0;
    for (int m = 0; m < n; ++m)
    {
      oenergy ef;
      oracle_cbmc_framework_molecule(p->ff, &p->box, p->grids, p->gnx, p->gny, p->gnz, &p->grid_cell, p->framework,
                                        p->n_framework,
                                     p->ff->cutoff_framework_vdw, p->ff->cutoff_coulomb, &atoms[m * na], na, -1, &ef);
      e += ef.framework_molecule_vdw + ef.framework_molecule_charge;
      if (m + 1 < n)
      {
        oenergy em;
        oracle_cbmc_intermolecular(p->ff, &p->box, &atoms[(m + 1) * na], (n - m - 1) * na, p->ff->cutoff_molecule_vdw,
                                   p->ff->cutoff_coulomb, &atoms[m * na], na, -1, -1, &em);
        e += em.molecule_molecule_vdw + em.molecule_molecule_charge;
      }
    }
    if (p->use_ewald && n > 0)
    {
      std::vector<int32_t> sizes(n, na);
      oenergy ee;
      oracle_ewald_fourier_energy(p->ff, &p->box, p->s_framework, atoms.data(), n * na, sizes.data(), n, 0.0, nullptr,
                                  &ee);
      e += ee.ewald_fourier + ee.ewald_self + ee.ewald_exclusion;
    }
    return e;
  }
};
}  // namespace

extern "C" void oracle_mixture_run(const omix_setup* setup, const double* xyz_in, const int32_t* comp_in, int n_in,
                                   int64_t steps, uint64_t seed, omix_result* out, double* xyz_out,
                                   int32_t* comp_out, double* seconds)
{
  Mixture mx(setup, seed * 0x100000001b3ULL + 0x51ed270b27ULL);
  const int na = mx.na;
  // inverse of the cell (columns = lattice vectors) for the minimum image of intramolecular separations
  const double(&h)[3][3] = mx.cell;  // h[c][r]: component r of lattice vector c
  const double det = h[0][0] * (h[1][1] * h[2][2] - h[1][2] * h[2][1]) - h[1][0] * (h[0][1] * h[2][2] - h[0][2] * h[2][1]) +
                     h[2][0] * (h[0][1] * h[1][2] - h[0][2] * h[1][1]);
  double M[3][3], inv[3][3];  // M[r][c] = h[c][r]; inv = M^-1: fractional k = sum_r inv[k][r] * cartesian r
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) M[r][c] = h[c][r];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      // inv[i][j] = cofactor(j, i) / det, cofactors from cyclic indices
      const int j1 = (j + 1) % 3, j2 = (j + 2) % 3, i1 = (i + 1) % 3, i2 = (i + 2) % 3;
      inv[i][j] = (M[j1][i1] * M[j2][i2] - M[j1][i2] * M[j2][i1]) / det;
    }
  for (int m = 0; m < n_in; ++m)
  {
    const omix_component& c = setup->comps[comp_in[m]];
    const double* r0 = xyz_in + 3 * (m * na);
    for (int i = 0; i < na; ++i)
    {
      // molecules are kept whole: atom i = atom 0 + the minimum image of their separation
      const double* ri = xyz_in + 3 * (m * na + i);
      const double dr[3] = {ri[0] - r0[0], ri[1] - r0[1], ri[2] - r0[2]};
      double sd[3];
      for (int k = 0; k < 3; ++k)
      {
        sd[k] = inv[k][0] * dr[0] + inv[k][1] * dr[1] + inv[k][2] * dr[2];
        sd[k] -= std::nearbyint(sd[k]);
      }
      oatom a{};
      a.x = r0[0] + h[0][0] * sd[0] + h[1][0] * sd[1] + h[2][0] * sd[2];
      a.y = r0[1] + h[0][1] * sd[0] + h[1][1] * sd[1] + h[2][1] * sd[2];
      a.z = r0[2] + h[0][2] * sd[0] + h[1][2] * sd[1] + h[2][2] * sd[2];
      a.charge = c.charges[i];
      a.scaling_vdw = a.scaling_coulomb = 1.0;
      a.molecule_id = static_cast<uint32_t>(m);
      a.type = static_cast<uint16_t>(c.types[i]);
      mx.atoms.push_back(a);
    }
    mx.comp.push_back(comp_in[m]);
    ++mx.count[comp_in[m]];
  }
  mx.n = n_in;
  // structure factors of the starting configuration (framework included), and its energy
  const int64_t nk = setup->use_ewald ? oracle_ewald_kvectors(setup->ff, &setup->box, nullptr, nullptr, nullptr) : 0;
  mx.stored.assign(10 * nk, 0.0);
  if (setup->use_ewald)
  {
    if (n_in > 0)
    {
      std::vector<int32_t> sizes(n_in, na);
      oenergy ee;
      oracle_ewald_fourier_energy(setup->ff, &setup->box, setup->s_framework, mx.atoms.data(), n_in * na,
                                  sizes.data(), n_in, 0.0, mx.stored.data(), &ee);
    }
    else
      for (int64_t k = 0; k < nk; ++k)
      {
        mx.stored[10 * k] = setup->s_framework ? setup->s_framework[2 * k] : 0.0;
        mx.stored[10 * k + 1] = setup->s_framework ? setup->s_framework[2 * k + 1] : 0.0;
      }
  }
  mx.energy = mx.recompute();
  // *seconds covers the moves only (not the set-up and final recomputations)
  const auto t0 = std::chrono::steady_clock::now();
  omix_result& r = *out;
  std::memset(&r, 0, sizeof(r));
  const double ptot = setup->p_translation + setup->p_rotation + setup->p_swap + setup->p_identity;
  for (int64_t s = 0; s < steps; ++s)
  {
    const int c = std::min(setup->n_components - 1, static_cast<int>(mx.rng.uniform() * setup->n_components));
    const double u = mx.rng.uniform() * ptot;
    int kind, acc;
    if (u < setup->p_translation)
    {
      kind = 0;
      acc = mx.translateOrRotate(c, false);
    }
    else if (u < setup->p_translation + setup->p_rotation)
    {
      kind = 1;
      acc = mx.translateOrRotate(c, true);
    }
    else if (u < setup->p_translation + setup->p_rotation + setup->p_swap)
    {
      if (mx.rng.uniform() < 0.5)
      {
        kind = 2;
        acc = mx.insertion(c);
      }
      else
      {
        kind = 3;
        acc = mx.deletion(c);
      }
    }
    else
    {
      kind = 4;
      acc = mx.identityChange(c);
    }
    r.attempted[kind] += 1;
    r.accepted[kind] += acc;
    for (int k = 0; k < setup->n_components; ++k) r.sum_n[k] += mx.count[k];
    r.samples += 1;
  }
  const auto t1 = std::chrono::steady_clock::now();
  for (int k = 0; k < 4; ++k) r.n_molecules[k] = mx.count[k];
  r.running_energy = mx.energy;
  r.recomputed_energy = mx.recompute();
  if (xyz_out)
    for (int i = 0; i < mx.n * na; ++i)
    {
      xyz_out[3 * i] = mx.atoms[i].x;
      xyz_out[3 * i + 1] = mx.atoms[i].y;
      xyz_out[3 * i + 2] = mx.atoms[i].z;
    }
  if (comp_out)
    for (int m = 0; m < mx.n; ++m) comp_out[m] = mx.comp[m];
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
}

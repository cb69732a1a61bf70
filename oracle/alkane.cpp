// FP64 CPU GCMC of flexible united-atom alkanes — TEST INFRASTRUCTURE ONLY.
//
// Restates, for linear chains grown from bead 0, the reference's configurational-bias growth of flexible molecules:
//   first bead        cbmc/multiple_first_bead.cpp:20-76 (k uniform positions; retrace keeps trial 0 at the old bead)
//   chain growth      cbmc/flexible_molecules/insertion.cpp:32-126 and deletion.cpp:30-104
//   trial generation  cbmc/operators.cpp:951-1078: the seed step (fixed bond length, uniform direction), and for every
//                     later bead one base conformation from generateFlexibleBaseConformation (:203-447, cold start:
//                     the bend angle drawn by BendPotential::generateBendAngle, bend_potential.cpp:197-220, then
//                     2*2*moves-per-open-bead internal Metropolis moves: bond-length change 0.3 (a fixed bond only
//                     draws its bead), bend-angle change 0.7 with the sine Jacobian) and per direction the
//                     coupled-decoupled torsion selection selectTorsionOrientation (:135-196)
//   moves             mc_moves/component/translation.cpp:30-200, insertion_cbmc.cpp:34-207 (Pacc = beta f V / (N+1)
//                     W / W_IG), deletion_cbmc.cpp:34-195 (Pacc = N / (beta f V) W_IG / W)
//   energies          potentialVDW<0> Lennard-Jones (potentials/pair_vdw.ixx:85-101) over the framework
//                     (cbmc/interactions_framework_molecule.cpp:31-104) and the other molecules
//                     (cbmc/interactions_intermolecular.cpp:22-95), overlap = a pair above the overlap criterion;
//                     harmonic bend (bend_potential.cpp:321-380), TraPPE torsion (torsion_potential.cpp:393-476),
//                     intra-molecular Lennard-Jones without cut-off between beads four or more bonds apart
//                     (van_der_waals_potential.cpp:43-62)
// Independent systems run in parallel (OpenMP), one system per thread.
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
using oracle_rng::Rng;
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kMinimumRosenbluth = 1e-150;  // forcefield.ixx:143

struct V3
{
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalized(V3 a) { return (1.0 / length(a)) * a; }

// double3::angle (mathkit/double3.ixx): atan2(|Rab x Rcb|, Rab . Rcb)
inline double angle(V3 a, V3 b, V3 c)
{
  const V3 rab = a - b, rcb = c - b;
  return std::atan2(length(cross(rab, rcb)), dot(rab, rcb));
}

// double3::rotateAroundAxis (mathkit/double3.ixx:163-178), axis = *this (a unit vector)
inline V3 rotateAroundAxis(V3 axis, V3 v, double ang)
{
  const double c = std::cos(ang), w = 1.0 - c;
  double s = std::sqrt(1.0 - c * c);
  if (ang < 0.0) s = -s;
  const double x = axis.x, y = axis.y, z = axis.z;
  return {v.x * (x * x * w + c) + v.y * (x * y * w + z * s) + v.z * (x * z * w - y * s),
          v.x * (x * y * w - z * s) + v.y * (y * y * w + c) + v.z * (y * z * w + x * s),
          v.x * (x * z * w + y * s) + v.y * (y * z * w - x * s) + v.z * (z * z * w + c)};
}

// RandomNumber::randomVectorOnUnitSphere (mathkit/randomnumbers.cpp:61-74)
V3 randomVectorOnUnitSphere(Rng& r)
{
  double r1, r2, sq;
  do
  {
    r1 = 2.0 * r.uniform() - 1.0;
    r2 = 2.0 * r.uniform() - 1.0;
    sq = r1 * r1 + r2 * r2;
  } while (sq >= 1.0);
  const double h = 2.0 * std::sqrt(1.0 - sq);
  return {r1 * h, r2 * h, 1.0 - 2.0 * sq};
}

// RandomNumber::randomVectorOnCone (mathkit/randomnumbers.cpp:77-86)
V3 randomVectorOnCone(Rng& r, V3 v, double ang)
{
  const V3 n = normalized(v);
  V3 w = randomVectorOnUnitSphere(r);
  w = w - dot(n, w) * n;
  return normalized(std::sin(ang) * normalized(w) + std::cos(ang) * n);
}

// CBMC::selectTrialPosition (cbmc/util.cpp:14-47)
int selectTrial(const std::vector<double>& logBF, double u)
{
  return oracle_select_trial(logBF.data(), static_cast<int>(logBF.size()), u);
}

struct Cell
{
  double c[3][3], ic[3][3];  // c[col][row]
  bool triclinic;
  double volume;
};

Cell makeCell(const obox& b)
{
  Cell k{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) k.c[c][r] = b.cell[3 * c + r];
  const double m11 = k.c[0][0], m12 = k.c[1][0], m13 = k.c[2][0];
  const double m21 = k.c[0][1], m22 = k.c[1][1], m23 = k.c[2][1];
  const double m31 = k.c[0][2], m32 = k.c[1][2], m33 = k.c[2][2];
  const double det = m11 * (m22 * m33 - m23 * m32) - m12 * (m21 * m33 - m23 * m31) + m13 * (m21 * m32 - m22 * m31);
  // inverse, stored in the same column convention (ic[col][row])
  const double inv[3][3] = {{(m22 * m33 - m32 * m23) / det, -(m12 * m33 - m32 * m13) / det,
                             (m12 * m23 - m22 * m13) / det},
                            {-(m21 * m33 - m31 * m23) / det, (m11 * m33 - m31 * m13) / det,
                             -(m11 * m23 - m21 * m13) / det},
                            {(m21 * m32 - m31 * m22) / det, -(m11 * m32 - m31 * m12) / det,
                             (m11 * m22 - m21 * m12) / det}};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) k.ic[c][r] = inv[r][c];
  k.triclinic = b.triclinic != 0;
  k.volume = det;
  return k;
}

inline double roundHalfAway(double x) { return static_cast<double>(static_cast<long>(x + (x >= 0 ? 0.5 : -0.5))); }

// SimulationBox::applyPeriodicBoundaryConditions (simulationbox.ixx:131-161)
inline V3 pbc(const Cell& b, V3 d)
{
  if (!b.triclinic)
    return {d.x - roundHalfAway(d.x * b.ic[0][0]) * b.c[0][0], d.y - roundHalfAway(d.y * b.ic[1][1]) * b.c[1][1],
            d.z - roundHalfAway(d.z * b.ic[2][2]) * b.c[2][2]};
  double s[3];
  const double v[3] = {d.x, d.y, d.z};
  for (int r = 0; r < 3; ++r) s[r] = b.ic[0][r] * v[0] + b.ic[1][r] * v[1] + b.ic[2][r] * v[2];
  for (int r = 0; r < 3; ++r) s[r] -= roundHalfAway(s[r]);
  return {b.c[0][0] * s[0] + b.c[1][0] * s[1] + b.c[2][0] * s[2],
          b.c[0][1] * s[0] + b.c[1][1] * s[1] + b.c[2][1] * s[2],
          b.c[0][2] * s[0] + b.c[1][2] * s[1] + b.c[2][2] * s[2]};
}

// potentialVDW<0> Lennard-Jones at full scaling (potentials/pair_vdw.ixx:85-101)
inline double pairLJ(const off* ff, int ta, int tb, double rr)
{
  const int idx = ta * ff->n_types + tb;
  if (!ff->lj[idx]) return 0.0;
  const double arg1 = 4.0 * ff->epsilon[idx];
  const double arg2 = ff->sigma[idx] * ff->sigma[idx];
  const double temp = rr / arg2;
  const double rri3 = 1.0 / (temp * temp * temp);
  return arg1 * (rri3 * (rri3 - 1.0)) - ff->shift[idx];
}

// The intra-molecular potentials of a linear chain
struct Intra
{
  const off* ff;
  const oalkane* c;

  // BendPotential::calculateEnergy, harmonic (bend_potential.cpp:321-380)
  double bend(V3 a, V3 b, V3 cc) const
  {
    V3 ab = a - b, cb = cc - b;
    ab = (1.0 / std::sqrt(dot(ab, ab))) * ab;
    cb = (1.0 / std::sqrt(dot(cb, cb))) * cb;
    const double ct = std::clamp(dot(ab, cb), -1.0, 1.0);
    const double theta = std::acos(ct);
    return 0.5 * c->bend_k * (theta - c->bend_theta0) * (theta - c->bend_theta0);
  }

  // TorsionPotential::calculateEnergy, TraPPE (torsion_potential.cpp:393-476)
  double torsion(V3 a, V3 b, V3 cc, V3 d) const
  {
    const V3 dab = a - b;
    const V3 dcb = normalized(cc - b);
    const V3 ddc = d - cc;
    const double dot_ab = dot(dab, dcb), dot_dc = dot(ddc, dcb);
    const V3 dr = normalized(dab - dot_ab * dcb);
    const V3 ds = normalized(ddc - dot_dc * dcb);
    const double cp = std::clamp(dot(dr, ds), -1.0, 1.0);
    const double* p = c->torsion;
    return p[0] + (1.0 + cp) * (p[1] + p[3] - 2.0 * (cp - 1.0) * (p[2] - 2.0 * p[3] * cp));
  }

  // intra-molecular Lennard-Jones between bead j and beads i <= j - 4 (no cut-off, scaling 1)
  double vdwOf(const V3* x, int j) const
  {
    double e = 0.0;
    for (int i = 0; i + 4 <= j; ++i)
    {
      const V3 d = x[j] - x[i];
      const double rr = dot(d, d);
      const int idx = c->types[i] * ff->n_types + c->types[j];
      const double s2 = ff->sigma[idx] * ff->sigma[idx];
      const double rri = s2 / rr;
      const double t = rri * rri * rri;
      e += 4.0 * ff->epsilon[idx] * (t * (t - 1.0));
    }
    return e;
  }

  // all internal terms of a chain (IntraMolecularPotentials::computeInternalEnergies; bonds are fixed)
  double total(const V3* x) const
  {
    double e = 0.0;
    const int nb = c->n_beads;
    for (int j = 2; j < nb; ++j) e += bend(x[j - 2], x[j - 1], x[j]);
    for (int j = 3; j < nb; ++j) e += torsion(x[j - 3], x[j - 2], x[j - 1], x[j]);
    for (int j = 4; j < nb; ++j) e += vdwOf(x, j);
    return e;
  }

  // BendPotential::generateBendAngle, harmonic (bend_potential.cpp:208-220)
  double generateBendAngle(Rng& r, double beta) const
  {
    double theta, s, e;
    do
    {
      theta = kPi * r.uniform();
      s = std::sin(theta);
      e = 0.5 * c->bend_k * (theta - c->bend_theta0) * (theta - c->bend_theta0);
    } while (r.uniform() > (s * s) * std::exp(-beta * e));
    return theta;
  }

  // generateFlexibleBaseConformation (operators.cpp:203-447) for one next bead j with previous j-2, current j-1,
  // one bend and a fixed bond; cold start (empty conformation reservoir)
  V3 baseConformation(Rng& r, double beta, const V3* x, int j) const
  {
    const V3 prev = x[j - 2], cur = x[j - 1];
    const V3 last = normalized(prev - cur);
    const double ang0 = generateBendAngle(r, beta);
    V3 nxt = cur + c->bond_length * randomVectorOnCone(r, last, ang0);
    const int trials = 2 * c->n_moves_per_open_bead * 1 * 2;
    double bendE = bend(prev, cur, nxt);
    for (int t = 0; t < trials; ++t)
    {
      // categoricalDistribution({0.3, 0.7, 0.0})
      const bool bondMove = r.uniform() < 0.3;
      if (bondMove)
      {
        (void)r.uniform();  // selects the bead; a fixed bond is not changed
        continue;
      }
      // bend-angle change (operators.cpp:369-407)
      (void)r.uniform();  // selects the bead
      const double curAngle = angle(prev, cur, nxt);
      const double curSin = std::sin(curAngle);
      const V3 dr = cur - nxt;
      const V3 perp = normalized(cross(dr, last));
      const double ra = (2.0 * r.uniform() - 1.0) * 0.3;  // bendAngleChange.maxChange
      const V3 bv = nxt - cur;
      const V3 trial = cur + rotateAroundAxis(perp, bv, ra);
      const double newSin = std::sin(angle(prev, cur, trial));
      const double newE = bend(prev, cur, trial);
      if (r.uniform() < (newSin / curSin) * std::exp(-beta * (newE - bendE)))
      {
        nxt = trial;
        bendE = newE;
      }
    }
    return nxt;
  }

  // selectTorsionOrientation (operators.cpp:135-196) for one next bead j; returns the position and the torsion weight
  V3 torsionSelect(Rng& r, double beta, const V3* x, int j, V3 base, bool pinFirst, double& weight) const
  {
    const int n = c->n_torsion_trials;
    const V3 cur = x[j - 1];
    const V3 last = normalized(x[j - 2] - cur);
    std::vector<V3> pos(n);
    std::vector<double> logBF(n);
    for (int s = 0; s < n; ++s)
    {
      const double a = (pinFirst && s == 0) ? 0.0 : (2.0 * r.uniform() - 1.0) * kPi;
      pos[s] = cur + rotateAroundAxis(last, base - cur, a);
      const double e = j >= 3 ? torsion(x[j - 3], x[j - 2], cur, pos[s]) : 0.0;
      logBF[s] = -beta * e;
    }
    double w = 0.0;
    for (double l : logBF) w += std::exp(l);
    weight = w / static_cast<double>(n);
    const int sel = pinFirst ? 0 : selectTrial(logBF, r.uniform());
    return pos[sel];
  }
};

struct SystemState
{
  const oalkane_setup* p;
  const off* ff;
  Rng rng;
  Cell cell;
  Intra intra;
  int nb;
  std::vector<V3> fw;
  std::vector<int> fwType;
  std::vector<V3> mol;  // n * nb positions
  int n = 0;
  double energy = 0.0;

  SystemState(const oalkane_setup* setup, uint64_t seed)
      : p(setup), ff(setup->ff), rng(seed), cell(makeCell(setup->box)), intra{setup->ff, &setup->chain},
        nb(setup->chain.n_beads)
  {
    for (int a = 0; a < setup->n_framework; ++a)
    {
      fw.push_back({setup->framework[a].x, setup->framework[a].y, setup->framework[a].z});
      fwType.push_back(setup->framework[a].type);
    }
  }

  V3 randomPosition()
  {
    // SimulationBox::randomPosition (simulationbox.cpp:132-135)
    const double s0 = rng.uniform(), s1 = rng.uniform(), s2 = rng.uniform();
    return {cell.c[0][0] * s0 + cell.c[1][0] * s1 + cell.c[2][0] * s2,
            cell.c[0][1] * s0 + cell.c[1][1] * s1 + cell.c[2][1] * s2,
            cell.c[0][2] * s0 + cell.c[1][2] * s1 + cell.c[2][2] * s2};
  }

  // external energy of one bead of type t at r, against the framework and every molecule but `skip`
  bool bead(V3 r, int t, int skip, double& efw, double& emm) const
  {
    const double overlap = ff->overlap_criteria;
    const double rcf = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
    const double rcm = ff->cutoff_molecule_vdw * ff->cutoff_molecule_vdw;
    efw = emm = 0.0;
    for (std::size_t a = 0; a < fw.size(); ++a)
    {
      const V3 d = pbc(cell, fw[a] - r);
      const double rr = dot(d, d);
      if (rr < rcf)
      {
        const double e = pairLJ(ff, fwType[a], t, rr);
        if (e > overlap) return false;
        efw += e;
      }
    }
    for (int m = 0; m < n; ++m)
    {
      if (m == skip) continue;
      for (int b = 0; b < nb; ++b)
      {
        const V3 d = pbc(cell, mol[m * nb + b] - r);
        const double rr = dot(d, d);
        if (rr < rcm)
        {
          const double e = pairLJ(ff, p->chain.types[b], t, rr);
          if (e > overlap) return false;
          emm += e;
        }
      }
    }
    return true;
  }

  // One growth (retrace when m >= 0: the old positions of molecule m are trial 0 of every step).
  // Returns false when every trial of a step overlaps or the chain weight falls below the minimum.
  bool grow(int m, std::vector<V3>& x, double& W, double& eext)
  {
    const oalkane& c = p->chain;
    const double beta = p->beta;
    const bool retrace = m >= 0;
    const V3* old = retrace ? &mol[m * nb] : nullptr;
    const int skip = retrace ? m : -1;
    x.assign(nb, V3{0, 0, 0});

    // first bead (multiple_first_bead.cpp:20-76)
    const int k1 = c.n_first_bead_trials;
    std::vector<V3> tr(k1);
    for (int t = 0; t < k1; ++t) tr[t] = (retrace && t == 0) ? old[0] : randomPosition();
    std::vector<double> logBF, ext;
    std::vector<int> idx;
    for (int t = 0; t < k1; ++t)
    {
      double f, mm;
      if (!bead(tr[t], c.types[0], skip, f, mm)) continue;
      logBF.push_back(-beta * (f + mm));
      ext.push_back(f + mm);
      idx.push_back(t);
    }
    if (logBF.empty() || (retrace && idx[0] != 0)) return false;
    double w = 0.0;
    for (double l : logBF) w += std::exp(l);
    W = w / static_cast<double>(k1);
    int sel = retrace ? 0 : selectTrial(logBF, rng.uniform());
    x[0] = tr[idx[sel]];
    eext = ext[sel];

    // chain (flexible_molecules/insertion.cpp:32-126, deletion.cpp:30-104)
    double Wc = 1.0;
    const int kd = c.n_trial_directions;
    std::vector<V3> dir(kd);
    std::vector<double> tw(kd);
    for (int j = 1; j < nb; ++j)
    {
      if (j == 1)
      {
        // seed step (operators.cpp:994-1004 / 1050-1061): fixed bond length, uniform direction
        for (int i = 0; i < kd; ++i)
        {
          tw[i] = 1.0;
          dir[i] = (retrace && i == 0) ? old[1] : x[0] + c.bond_length * randomVectorOnUnitSphere(rng);
        }
      }
      else if (!retrace)
      {
        // one shared base conformation, one torsion selection per direction (operators.cpp:1006-1013)
        const V3 base = intra.baseConformation(rng, beta, x.data(), j);
        for (int i = 0; i < kd; ++i) dir[i] = intra.torsionSelect(rng, beta, x.data(), j, base, false, tw[i]);
      }
      else
      {
        // retrace: the old orientation is the base of every direction and torsion trial 0 of direction 0
        // (operators.cpp:1064-1077)
        for (int i = 0; i < kd; ++i)
        {
          const V3 pos = intra.torsionSelect(rng, beta, old, j, old[j], i == 0, tw[i]);
          dir[i] = i == 0 ? old[j] : pos;
        }
      }
      logBF.clear();
      ext.clear();
      idx.clear();
      for (int i = 0; i < kd; ++i)
      {
        double f, mm;
        if (!bead(dir[i], c.types[j], skip, f, mm)) continue;
        x[j] = dir[i];
        const double eIntra = intra.vdwOf(x.data(), j);
        logBF.push_back(-beta * (f + mm + eIntra));
        ext.push_back(f + mm);
        idx.push_back(i);
      }
      if (logBF.empty() || (retrace && idx[0] != 0)) return false;
      w = 0.0;
      for (double l : logBF) w += std::exp(l);
      sel = retrace ? 0 : selectTrial(logBF, rng.uniform());
      Wc *= tw[idx[sel]] * w / static_cast<double>(kd);
      if (!retrace && Wc < kMinimumRosenbluth) return false;
      x[j] = dir[idx[sel]];
      eext += ext[sel];
    }
    W *= Wc;
    return true;
  }

  int translation()
  {
    if (n == 0) return 0;
    const int m = std::min(n - 1, static_cast<int>(rng.uniform() * n));
    const int dir = std::min(2, static_cast<int>(3.0 * rng.uniform()));
    const double disp = p->max_translation * 2.0 * (rng.uniform() - 0.5);
    V3 dv{0, 0, 0};
    (&dv.x)[dir] = disp;
    double eNew = 0.0, eOld = 0.0;
    for (int b = 0; b < nb; ++b)
    {
      double f, mm;
      if (!bead(mol[m * nb + b] + dv, p->chain.types[b], m, f, mm)) return 0;
      eNew += f + mm;
    }
    for (int b = 0; b < nb; ++b)
    {
      double f, mm;
      bead(mol[m * nb + b], p->chain.types[b], m, f, mm);
      eOld += f + mm;
    }
    const double dU = eNew - eOld;
    if (rng.uniform() < std::exp(-p->beta * dU))
    {
      for (int b = 0; b < nb; ++b) mol[m * nb + b] = mol[m * nb + b] + dv;
      energy += dU;
      return 1;
    }
    return 0;
  }

  int insertion()
  {
    if (n >= p->max_molecules) return 0;
    std::vector<V3> x;
    double W, eext;
    if (!grow(-1, x, W, eext)) return 0;
    const double pacc = p->beta * p->fugacity * cell.volume / static_cast<double>(n + 1) * W / p->w_ig;
    if (rng.uniform() < pacc)
    {
      mol.insert(mol.end(), x.begin(), x.end());
      ++n;
      energy += eext + intra.total(x.data());
      return 1;
    }
    return 0;
  }

  int deletion()
  {
    if (n == 0) return 0;
    const int m = std::min(n - 1, static_cast<int>(rng.uniform() * n));
    std::vector<V3> x;
    double W, eext;
    if (!grow(m, x, W, eext)) return 0;
    const double pacc = static_cast<double>(n) / (p->beta * p->fugacity * cell.volume) * p->w_ig / W;
    if (rng.uniform() < pacc)
    {
      energy -= eext + intra.total(&mol[m * nb]);
      if (m != n - 1) std::copy(mol.begin() + (n - 1) * nb, mol.begin() + n * nb, mol.begin() + m * nb);
      mol.resize((n - 1) * nb);
      --n;
      return 1;
    }
    return 0;
  }

  void energies(double out[3]) const
  {
    out[0] = out[1] = out[2] = 0.0;
    SystemState& self = const_cast<SystemState&>(*this);
    const int n0 = n;
    for (int m = 0; m < n0; ++m)
    {
      out[2] += intra.total(&mol[m * nb]);
      for (int b = 0; b < nb; ++b)
      {
        // framework part, and the molecules after m (each pair once)
        double f, mm;
        self.n = 0;
        bead(mol[m * nb + b], p->chain.types[b], -1, f, mm);
        self.n = n0;
        out[0] += f;
        const double rcm = ff->cutoff_molecule_vdw * ff->cutoff_molecule_vdw;
        for (int m2 = m + 1; m2 < n0; ++m2)
          for (int b2 = 0; b2 < nb; ++b2)
          {
            const V3 d = pbc(cell, mol[m2 * nb + b2] - mol[m * nb + b]);
            const double rr = dot(d, d);
            if (rr < rcm) out[1] += pairLJ(ff, p->chain.types[b2], p->chain.types[b], rr);
          }
      }
    }
  }
};
}  // namespace

extern "C" void oracle_alkane_run(const oalkane_setup* setups, int n_systems, int64_t steps, int64_t equilibration,
                                  uint64_t seed, int threads, ogcmc_result* out, double* xyz, double* seconds,
                                  const double* xyz_in, const int32_t* n_in)
{
  std::vector<int64_t> offset(n_systems + 1, 0);
  for (int s = 0; s < n_systems; ++s)
    offset[s + 1] = offset[s] + static_cast<int64_t>(setups[s].max_molecules) * setups[s].chain.n_beads * 3;
  auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
  for (int s = 0; s < n_systems; ++s)
  {
    const oalkane_setup* p = &setups[s];
    SystemState st(p, seed * 0x100000001b3ULL + static_cast<uint64_t>(s) * 0x9e3779b97f4a7c15ULL + 7);
    if (n_in && n_in[s] > 0)
    {
      const double* q = xyz_in + offset[s];
      for (int i = 0; i < n_in[s] * st.nb; ++i) st.mol.push_back({q[3 * i], q[3 * i + 1], q[3 * i + 2]});
      st.n = n_in[s];
      double e[3];
      st.energies(e);
      st.energy = e[0] + e[1] + e[2];
    }
    ogcmc_result& r = out[s];
    std::memset(&r, 0, sizeof(r));
    const double ptot = p->p_translation + p->p_swap;
    const int64_t block = steps / 5 > 0 ? steps / 5 : 1;
    double block_sum = 0.0;
    int64_t block_cnt = 0;
    int bi = 0;
    for (int64_t k = 0; k < equilibration + steps; ++k)
    {
      int kind, acc;
      if (st.rng.uniform() * ptot < p->p_translation)
      {
        kind = 0;
        acc = st.translation();
      }
      else if (st.rng.uniform() < 0.5)
      {
        kind = 2;
        acc = st.insertion();
      }
      else
      {
        kind = 3;
        acc = st.deletion();
      }
      if (k >= equilibration)
      {
        r.attempted[kind] += 1;
        r.accepted[kind] += acc;
        r.sum_n += st.n;
        r.sum_n2 += static_cast<double>(st.n) * st.n;
        r.sum_energy += st.energy;
        r.samples += 1;
        block_sum += st.n;
        if (++block_cnt == block && bi < 5)
        {
          r.block_n[bi++] = block_sum / static_cast<double>(block_cnt);
          block_sum = 0.0;
          block_cnt = 0;
        }
      }
    }
    r.n_molecules = st.n;
    r.running_energy = st.energy;
    double e[3];
    st.energies(e);
    r.recomputed_energy = e[0] + e[1] + e[2];
    if (xyz)
    {
      double* o = xyz + offset[s];
      for (int i = 0; i < st.n * st.nb; ++i)
      {
        o[3 * i] = st.mol[i].x;
        o[3 * i + 1] = st.mol[i].y;
        o[3 * i + 2] = st.mol[i].z;
      }
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
}

extern "C" void oracle_alkane_grow_vacuum(const off* ff, const oalkane* chain, double beta, int64_t n, uint64_t seed,
                                          int threads, double* w, double* theta, double* cos_phi)
{
  oalkane_setup setup{};
  setup.ff = ff;
  for (int d = 0; d < 3; ++d) setup.box.cell[4 * d] = 100.0;
  setup.chain = *chain;
  setup.beta = beta;
  setup.fugacity = 1.0;
  setup.w_ig = 1.0;
  const int nb = chain->n_beads;
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num(), nt = omp_get_num_threads();
#else
    const int tid = 0, nt = 1;
#endif
    SystemState st(&setup, seed * 0x100000001b3ULL + static_cast<uint64_t>(tid) * 0x9e3779b97f4a7c15ULL + 11);
    std::vector<V3> x;
    for (int64_t i = tid; i < n; i += nt)
    {
      double W = 0.0, e;
      if (!st.grow(-1, x, W, e)) W = 0.0;
      w[i] = W;
      if (W > 0.0)
      {
        for (int j = 2; theta && j < nb; ++j) theta[i * (nb - 2) + j - 2] = angle(x[j - 2], x[j - 1], x[j]);
        for (int j = 3; cos_phi && j < nb; ++j)
        {
          const V3 dab = x[j - 3] - x[j - 2], dcb = normalized(x[j - 1] - x[j - 2]), ddc = x[j] - x[j - 1];
          const V3 dr = normalized(dab - dot(dab, dcb) * dcb), ds = normalized(ddc - dot(ddc, dcb) * dcb);
          cos_phi[i * (nb - 3) + j - 3] = dot(dr, ds);
        }
      }
    }
  }
}

extern "C" void oracle_alkane_energy(const oalkane_setup* setup, const double* xyz, int n_molecules, double out[3])
{
  SystemState st(setup, 1);
  for (int i = 0; i < n_molecules * st.nb; ++i) st.mol.push_back({xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
  st.n = n_molecules;
  st.energies(out);
}

extern "C" void oracle_alkane_bead_energies(const oalkane_setup* setup, const double* xyz, int n_molecules,
                                            const double* xyz_beads, const int32_t* types, int n_beads, int skip,
                                            double* fw, double* mm, int32_t* overlap)
{
  SystemState st(setup, 1);
  for (int i = 0; i < n_molecules * st.nb; ++i) st.mol.push_back({xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]});
  st.n = n_molecules;
  for (int b = 0; b < n_beads; ++b)
  {
    const bool ok = st.bead({xyz_beads[3 * b], xyz_beads[3 * b + 1], xyz_beads[3 * b + 2]}, types[b], skip, fw[b],
                            mm[b]);
    overlap[b] = ok ? 0 : 1;
    if (!ok)
    {
      // the energies up to the first overlapping pair are not meaningful
      fw[b] = mm[b] = 0.0;
    }
  }
}

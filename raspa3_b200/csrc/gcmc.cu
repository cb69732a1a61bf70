// Device-resident grand-canonical Monte Carlo of rigid molecules: many independent chains, one CTA per chain.
//
// Each CTA runs a chain for a number of moves per launch, entirely on the device: the moves, energies, Rosenbluth
// weights and acceptance tests of the reference's
//   translation    src/raspakit/mc_moves/component/translation.cpp:30-200
//   rotation       src/raspakit/mc_moves/component/rotation.cpp:30-190
//   CBMC insertion src/raspakit/mc_moves/component/insertion_cbmc.cpp:34-207 (first beads: cbmc/multiple_first_bead.cpp
//                  :20-49; rigid orientations: cbmc/operators.cpp:951-970; selection: cbmc/util.cpp:14-47)
//   CBMC deletion  src/raspakit/mc_moves/component/deletion_cbmc.cpp:34-195 (retrace: cbmc/multiple_first_bead.cpp:51-76)
// with the framework-molecule energy from the tricubic grids, the molecule-molecule Lennard-Jones and real-space Ewald
// pair sums, and the Ewald Fourier energy change on the chain's own structure factors (which include the framework).
//
// Work split inside a CTA of 128 threads: the external energy of a set of trial atoms is one warp's job (lanes own the
// atoms' grid interpolations, then stride over the partner atoms; warp-shuffle reduction), four warps take four trial
// sets at a time; the Ewald change is spread over all threads by k-vector, from per-atom phase tables built in shared
// memory (e^{i 2 pi m s_d}, m = 0..kmax). All sums are in a fixed order (deterministic); arithmetic is FP64. Random
// numbers come from a counter-based generator (Philox-4x32-10, Salmon et al., SC'11) keyed by seed and chain and
// counted by (move, slot), so any thread can draw any move's numbers without shared state.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"
#include "rng.cuh"

namespace
{
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxAtoms = 8;     // atoms per molecule
constexpr int kMaxTrials = 16;   // first-bead positions / orientations per step
constexpr int kMaxK = 16;        // kmax per axis + 1 supported by the phase tables

struct Component
{
  int n_atoms;
  int starting_bead;
  int types[kMaxAtoms];
  double charges[kMaxAtoms];
  double masses[kMaxAtoms];
  double offsets[kMaxAtoms][3];
  double self_excl;  // Ewald self + exclusion energy one inserted molecule adds (ewald.cpp:1164-1238, new-atom terms)
};

struct Params
{
  rgd::FF ff;
  rgd::Box box;
  rgd::Grid grid;            // data unused; shape and inverse cell
  const double* vdw_grid[kMaxAtoms];  // grid of each component atom's type (NULL = no framework term)
  const double* ewald_grid;
  int quintic;  // the grids hold the 27 triquintic values per point (RG_SCHEME_TRIQUINTIC) instead of 8
  double rcv_fw2, rcv_mol2, rcc2;
  Component comp;
  double beta, fugacity, volume;
  double max_translation, max_rotation;
  double p_translation, p_rotation, p_swap;
  int k1, k2;
  int capacity;
  int use_ewald;
  int64_t nk;
  int kmax[3];
  const char4* kvec;
  const double* temp;
  unsigned long long seed;
  // learned first-bead proposal (null: uniform): inclusive cumulative cell probabilities and the density relative to
  // uniform, over G^3 cells of the unit cell; the simulation box is rep[0] x rep[1] x rep[2] unit cells
  const double* prop_cdf;
  const double* prop_q;
  int prop_G;
  double prop_eps;
  double uc[3][3];   // unit cell c[col][row]
  double uic[3][3];  // its inverse
  int rep[3];
  // per-chain state
  double4* pos;              // [chain][capacity * n_atoms]
  double2* sk;               // [chain][nk] structure factors (framework included)
  double2* dsk;              // [chain][nk] scratch: structure-factor change of the current move
  int* n;                    // [chain]
  double* energy;            // [chain]
  double* stats;             // [chain][kStats]
};

constexpr int kStats = 24;  // attempted[4], accepted[4], sum_n, sum_n2, sum_energy, samples, block_n[5] (sums), block_cnt

using rgd::philox;
using rgd::uniform2;

// random slots of one move
enum Slot
{
  kSlotMove = 0,       // (move kind, insertion-or-deletion)
  kSlotPick = 1,       // (molecule, direction)
  kSlotChange = 2,     // (displacement or angle, acceptance)
  kSlotSelect = 3,     // (first-bead selection, orientation selection)
  kSlotFirst = 16,     // + 4 t: first-bead position t (up to 8 numbers)
  kSlotOrient = 128    // + 2 t: orientation t (3 numbers)
};

__device__ __forceinline__ void rotationFromUniforms(double u1, double u2, double u3, double R[3][3])
{
  // uniform unit quaternion (Shoemake) -> rotation matrix
  const double x = sqrt(1 - u1) * sinpi(2 * u2), y = sqrt(1 - u1) * cospi(2 * u2);
  const double z = sqrt(u1) * sinpi(2 * u3), w = sqrt(u1) * cospi(2 * u3);
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

struct Shared
{
  double trial[kMaxTrials][kMaxAtoms][3];  // positions of the trial sets
  double setE[kMaxTrials];
  int setOv[kMaxTrials];
  double logq[kMaxTrials];
  double newPos[kMaxAtoms][3];
  double oldPos[kMaxAtoms][3];
  double red[kWarps];
  double u[8];
  int ints[8];
  double dbl[8];
};

// External energy (framework grids + other molecules) of `count` atoms at pos[], component atom indices atomIdx[],
// excluding molecule slot `skip`; evaluated by one warp. Returns the energy; *overlap set if the set overlaps.
template <bool QUINTIC>  // the system's grids: triquintic (27 values per point) or tricubic (8)
__device__ double warpExternal(const Params& p, int chain, int n, const double (*pos)[3], const int* atomIdx,
                               int count, int skip, int* overlap)
{
  const int lane = threadIdx.x & 31;
  double e = 0.0;
  int ov = 0;
  const Component& c = p.comp;
  // framework part: one lane per atom
  if (lane < count)
  {
    const int ai = atomIdx[lane];
    const double* g = p.vdw_grid[ai];
    if (g)
    {
      rgd::Grid gg = p.grid;
      gg.data = g;
      const double v = QUINTIC ? rgd::interpolateQuintic(gg, pos[lane][0], pos[lane][1], pos[lane][2], nullptr)
                               : rgd::interpolate(gg, pos[lane][0], pos[lane][1], pos[lane][2]);
      if (v > p.ff.overlap) ov = 1;
      e += v;
      if (p.ff.use_charge && p.ewald_grid)
      {
        gg.data = p.ewald_grid;
        e += c.charges[ai] * (QUINTIC ? rgd::interpolateQuintic(gg, pos[lane][0], pos[lane][1], pos[lane][2], nullptr)
                                      : rgd::interpolate(gg, pos[lane][0], pos[lane][1], pos[lane][2]));
      }
    }
  }
  // molecule-molecule part: lanes stride over partner atoms of the other molecules
  const int na = c.n_atoms;
  const double4* cpos = p.pos + static_cast<long long>(chain) * p.capacity * na;
  const int total = n * na;
  for (int q = lane; q < total; q += 32)
  {
    const int m = q / na, bj = q - m * na;
    if (m == skip) continue;
    const double4 B = cpos[q];
    const int tB = c.types[bj];
    const double qB = c.charges[bj];
    for (int i = 0; i < count; ++i)
    {
      const int ai = atomIdx[i];
      double dx = B.x - pos[i][0], dy = B.y - pos[i][1], dz = B.z - pos[i][2];
      rgd::pbc(p.box, dx, dy, dz);
      const double rr = dx * dx + dy * dy + dz * dz;
      if (rr < p.rcv_mol2)
      {
        const double2 f = rgd::pairVDW(p.ff, 1.0, 1.0, rr, tB, c.types[ai]);
        if (f.x > p.ff.overlap) ov = 1;
        e += f.x;
      }
      if (p.ff.use_charge && rr < p.rcc2) e += rgd::pairCoulomb(p.ff, 1.0, 1.0, sqrt(rr), qB, c.charges[ai]).x;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
  {
    e += __shfl_down_sync(0xffffffffu, e, o);
    ov |= __shfl_down_sync(0xffffffffu, ov, o);
  }
  *overlap = __shfl_sync(0xffffffffu, ov, 0);
  return __shfl_sync(0xffffffffu, e, 0);
}

// Ewald Fourier energy change of replacing the old atoms by the new ones (either may be absent); leaves the change of
// the structure factors in dsk. Block-wide; returns the energy on every thread.
__device__ double blockEwaldDelta(const Params& p, int chain, const double (*newPos)[3], int nNew,
                                  const double (*oldPos)[3], int nOld, double2* tab, double* red)
{
  const Component& c = p.comp;
  const int nAt = nNew + nOld;
  const int kx1 = p.kmax[0] + 1, ky1 = p.kmax[1] + 1, kz1 = p.kmax[2] + 1;
  const int stride = kx1 + ky1 + kz1;
  // phase tables e^{i 2 pi m s_d}
  for (int idx = threadIdx.x; idx < nAt * stride; idx += blockDim.x)
  {
    const int a = idx / stride, m = idx - a * stride;
    const double* r = a < nNew ? newPos[a] : oldPos[a - nNew];
    const int d = m < kx1 ? 0 : (m < kx1 + ky1 ? 1 : 2);
    const int mm = d == 0 ? m : (d == 1 ? m - kx1 : m - kx1 - ky1);
    const double s = p.box.ic[0][d] * r[0] + p.box.ic[1][d] * r[1] + p.box.ic[2][d] * r[2];
    double sn, cs;
    sincospi(2.0 * static_cast<double>(mm) * s, &sn, &cs);
    tab[idx] = make_double2(cs, sn);
  }
  __syncthreads();
  const double2* S = p.sk + static_cast<long long>(chain) * p.nk;
  double2* D = p.dsk + static_cast<long long>(chain) * p.nk;
  double e = 0.0;
  for (long long k = threadIdx.x; k < p.nk; k += blockDim.x)
  {
    const char4 kv = p.kvec[k];
    const int ay = abs(kv.y), az = abs(kv.z);
    const double sy = kv.y < 0 ? -1.0 : 1.0, sz = kv.z < 0 ? -1.0 : 1.0;
    double2 d = make_double2(0.0, 0.0);
    for (int a = 0; a < nAt; ++a)
    {
      const double2* t = tab + a * stride;
      const double2 ex = t[kv.x];
      double2 ey = t[kx1 + ay], ez = t[kx1 + ky1 + az];
      ey.y *= sy;
      ez.y *= sz;
      const double2 xy = make_double2(ex.x * ey.x - ex.y * ey.y, ex.x * ey.y + ex.y * ey.x);
      const double2 ph = make_double2(xy.x * ez.x - xy.y * ez.y, xy.x * ez.y + xy.y * ez.x);
      const double w = a < nNew ? c.charges[a] : -c.charges[a - nNew];
      d.x += w * ph.x;
      d.y += w * ph.y;
    }
    const double2 s = S[k];
    e += p.temp[k] * (2.0 * (s.x * d.x + s.y * d.y) + (d.x * d.x + d.y * d.y));
    D[k] = d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  double tot = 0.0;
  for (int w = 0; w < kWarps; ++w) tot += red[w];
  __syncthreads();
  return tot;
}

__device__ void blockAcceptEwald(const Params& p, int chain)
{
  double2* S = p.sk + static_cast<long long>(chain) * p.nk;
  const double2* D = p.dsk + static_cast<long long>(chain) * p.nk;
  for (long long k = threadIdx.x; k < p.nk; k += blockDim.x)
  {
    const double2 d = D[k];
    S[k].x += d.x;
    S[k].y += d.y;
  }
}

// CBMC::selectTrialPosition (cbmc/util.cpp:14-47) over the non-overlapping trials; returns the chosen trial index and
// the Rosenbluth weight sum_i exp(-beta U_i) / k, or -1 if every trial overlaps.
// With a proposal density, trial t's log weight is -beta U_t - log q_t (logq may be null: uniform, q = 1).
__device__ int selectTrial(const double* E, const int* ov, const double* logq, int k, double beta, double u, double* W)
{
  double largest = -1e300;
  bool any = false;
  for (int t = 0; t < k; ++t)
    if (!ov[t])
    {
      largest = fmax(largest, -beta * E[t] - (logq ? logq[t] : 0.0));
      any = true;
    }
  if (!any)
  {
    *W = 0.0;
    return -1;
  }
  double sum = 0.0, w = 0.0;
  for (int t = 0; t < k; ++t)
    if (!ov[t])
    {
      const double lw = -beta * E[t] - (logq ? logq[t] : 0.0);
      sum += exp(lw - largest);
      w += exp(lw);
    }
  *W = w / static_cast<double>(k);
  const double ws = u * sum;
  int first = -1, selected = -1;
  double cumw = 0.0;
  for (int t = 0; t < k; ++t)
  {
    if (ov[t]) continue;
    const double lw = -beta * E[t] - (logq ? logq[t] : 0.0);
    if (first < 0)
    {
      first = t;
      selected = t;
      cumw = exp(lw - largest);
      continue;
    }
    if (cumw < ws)
    {
      cumw += exp(lw - largest);
      selected = t;
    }
  }
  return selected;
}

// Proposal density (relative to uniform) of a position: the cell of its unit-cell fractional coordinates.
__device__ __forceinline__ double proposalDensity(const Params& p, const double r[3])
{
  int c[3];
  for (int a = 0; a < 3; ++a)
  {
    const double s = rgd::fract1(p.uic[0][a] * r[0] + p.uic[1][a] * r[1] + p.uic[2][a] * r[2]);
    c[a] = min(p.prop_G - 1, static_cast<int>(s * p.prop_G));
  }
  return p.prop_q[c[0] + p.prop_G * (c[1] + p.prop_G * c[2])];
}

extern __shared__ double2 gcmcDyn[];

template <bool QUINTIC>
__global__ void __launch_bounds__(kThreads) gcmcKernel(Params p, long long move0, int nmoves, int record,
                                                       long long block_len)
{
  const int chain = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ Shared sh;
  double2* tab = gcmcDyn;  // phase tables: 2 * kMaxAtoms atoms x (kx+ky+kz+3)
  const Component& c = p.comp;
  const int na = c.n_atoms;
  double4* cpos = p.pos + static_cast<long long>(chain) * p.capacity * na;
  double* st = p.stats + static_cast<long long>(chain) * kStats;
  const double ptot = p.p_translation + p.p_rotation + p.p_swap;

  for (int it = 0; it < nmoves; ++it)
  {
    const long long mv = move0 + it;
    const int n = p.n[chain];
    const double2 uMove = uniform2(p.seed, chain, mv, kSlotMove);
    const double2 uPick = uniform2(p.seed, chain, mv, kSlotPick);
    const double2 uChange = uniform2(p.seed, chain, mv, kSlotChange);
    const double x = uMove.x * ptot;
    const int kind = x < p.p_translation ? 0 : (x < p.p_translation + p.p_rotation ? 1 : (uMove.y < 0.5 ? 2 : 3));
    int accepted = 0;

    if (kind <= 1 && n > 0)
    {
      // ---- translation / rotation ----
      const int m = min(n - 1, static_cast<int>(uPick.x * n));
      const int dir = min(2, static_cast<int>(3.0 * uPick.y));
      if (threadIdx.x < na)
      {
        const int i = threadIdx.x;
        const double4 o = cpos[m * na + i];
        sh.oldPos[i][0] = o.x;
        sh.oldPos[i][1] = o.y;
        sh.oldPos[i][2] = o.z;
      }
      __syncthreads();
      if (threadIdx.x == 0)
      {
        if (kind == 0)
        {
          const double disp = p.max_translation * 2.0 * (uChange.x - 0.5);
          for (int i = 0; i < na; ++i)
            for (int d = 0; d < 3; ++d) sh.newPos[i][d] = sh.oldPos[i][d] + (d == dir ? disp : 0.0);
        }
        else
        {
          const double angle = p.max_rotation * 2.0 * (uChange.x - 0.5);
          const double cs = cos(angle), sn = sin(angle);
          double com[3] = {0, 0, 0}, wsum = 0.0;
          for (int i = 0; i < na; ++i)
          {
            for (int d = 0; d < 3; ++d) com[d] += c.masses[i] * sh.oldPos[i][d];
            wsum += c.masses[i];
          }
          for (int d = 0; d < 3; ++d) com[d] /= wsum;
          const int a = (dir + 1) % 3, b = (dir + 2) % 3;
          for (int i = 0; i < na; ++i)
          {
            double r[3] = {sh.oldPos[i][0] - com[0], sh.oldPos[i][1] - com[1], sh.oldPos[i][2] - com[2]};
            double q[3] = {r[0], r[1], r[2]};
            q[a] = cs * r[a] - sn * r[b];
            q[b] = sn * r[a] + cs * r[b];
            for (int d = 0; d < 3; ++d) sh.newPos[i][d] = com[d] + q[d];
          }
        }
      }
      __syncthreads();
      int idx[kMaxAtoms];
      for (int i = 0; i < kMaxAtoms; ++i) idx[i] = i;
      if (warp < 2)
      {
        int ov;
        const double e = warpExternal<QUINTIC>(p, chain, n, warp == 0 ? sh.newPos : sh.oldPos, idx, na, m, &ov);
        if (lane == 0)
        {
          sh.setE[warp] = e;
          sh.setOv[warp] = ov;
        }
      }
      __syncthreads();
      double dEw = 0.0;
      if (p.use_ewald) dEw = blockEwaldDelta(p, chain, sh.newPos, na, sh.oldPos, na, tab, sh.red);
      const double dU = sh.setE[0] - sh.setE[1] + dEw;
      accepted = (!sh.setOv[0]) && (uChange.y < exp(-p.beta * dU));
      if (accepted)
      {
        if (threadIdx.x < na)
          cpos[m * na + threadIdx.x] = make_double4(sh.newPos[threadIdx.x][0], sh.newPos[threadIdx.x][1],
                                                    sh.newPos[threadIdx.x][2], 0.0);
        if (p.use_ewald) blockAcceptEwald(p, chain);
        if (threadIdx.x == 0) p.energy[chain] += dU;
      }
    }
    else if (kind >= 2)
    {
      const bool insert = kind == 2;
      const bool retrace = !insert;
      if ((insert && n < p.capacity) || (retrace && n > 0))
      {
        const int m = insert ? n : min(n - 1, static_cast<int>(uPick.x * n));
        const int skip = insert ? -1 : m;
        const int sb = c.starting_bead;
        const double2 uSel = uniform2(p.seed, chain, mv, kSlotSelect);
        // first-bead trial positions (retrace: trial 0 is the existing first bead)
        for (int t = threadIdx.x; t < p.k1; t += blockDim.x)
        {
          if (retrace && t == 0)
          {
            const double4 o = cpos[m * na + sb];
            sh.trial[0][0][0] = o.x;
            sh.trial[0][0][1] = o.y;
            sh.trial[0][0][2] = o.z;
            continue;
          }
          const double2 a = uniform2(p.seed, chain, mv, kSlotFirst + 4 * t);
          const double2 b = uniform2(p.seed, chain, mv, kSlotFirst + 4 * t + 1);
          const double2 u = uniform2(p.seed, chain, mv, kSlotFirst + 4 * t + 2);
          if (!p.prop_cdf || u.x < p.prop_eps)
          {
            // SimulationBox::randomPosition (simulationbox.cpp:132-135)
            const double s0 = a.x, s1 = a.y, s2 = b.x;
            for (int r = 0; r < 3; ++r)
              sh.trial[t][0][r] = p.box.c[0][r] * s0 + p.box.c[1][r] * s1 + p.box.c[2][r] * s2;
          }
          else
          {
            // a cell of the tabulated proposal (binary search of the cumulative probabilities), a uniform point in
            // it, and a uniformly chosen unit-cell replica of the simulation box
            const double2 v = uniform2(p.seed, chain, mv, kSlotFirst + 4 * t + 3);
            const int G = p.prop_G;
            const int ncell = G * G * G;
            int lo = 0, hi = ncell - 1;
            while (lo < hi)
            {
              const int mid = (lo + hi) >> 1;
              if (p.prop_cdf[mid] < u.y)
                lo = mid + 1;
              else
                hi = mid;
            }
            const int ci = lo % G, cj = (lo / G) % G, ck = lo / (G * G);
            const double sf[3] = {(ci + a.x) / G + static_cast<double>(min(p.rep[0] - 1, static_cast<int>(b.y * p.rep[0]))),
                                  (cj + a.y) / G + static_cast<double>(min(p.rep[1] - 1, static_cast<int>(v.x * p.rep[1]))),
                                  (ck + b.x) / G + static_cast<double>(min(p.rep[2] - 1, static_cast<int>(v.y * p.rep[2])))};
            for (int r = 0; r < 3; ++r)
              sh.trial[t][0][r] = p.uc[0][r] * sf[0] + p.uc[1][r] * sf[1] + p.uc[2][r] * sf[2];
          }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < p.k1; t += blockDim.x)
          sh.logq[t] = p.prop_cdf ? log(proposalDensity(p, sh.trial[t][0])) : 0.0;
        int one[1] = {sb};
        for (int t = warp; t < p.k1; t += kWarps)
        {
          int ov;
          const double e = warpExternal<QUINTIC>(p, chain, n, sh.trial[t], one, 1, skip, &ov);
          if (lane == 0)
          {
            sh.setE[t] = e;
            sh.setOv[t] = ov;
          }
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
          double W1;
          int sel = selectTrial(sh.setE, sh.setOv, sh.logq, p.k1, p.beta, uSel.x, &W1);
          if (retrace) sel = sh.setOv[0] ? -1 : 0;
          sh.ints[0] = sel;
          sh.dbl[0] = W1;
          sh.dbl[1] = sel >= 0 ? sh.setE[sel] : 0.0;
          if (sel >= 0)
            for (int d = 0; d < 3; ++d) sh.dbl[2 + d] = sh.trial[sel][0][d];
        }
        __syncthreads();
        const int sel1 = sh.ints[0];
        if (sel1 >= 0)
        {
          const double W1 = sh.dbl[0], e1 = sh.dbl[1];
          const double fb[3] = {sh.dbl[2], sh.dbl[3], sh.dbl[4]};
          __syncthreads();
          // orientation trials about the first bead (retrace: trial 0 is the existing orientation)
          for (int t = threadIdx.x; t < p.k2; t += blockDim.x)
          {
            if (retrace && t == 0)
            {
              for (int i = 0; i < na; ++i)
              {
                const double4 o = cpos[m * na + i];
                sh.trial[0][i][0] = o.x;
                sh.trial[0][i][1] = o.y;
                sh.trial[0][i][2] = o.z;
              }
              continue;
            }
            const double2 a = uniform2(p.seed, chain, mv, kSlotOrient + 2 * t);
            const double2 b = uniform2(p.seed, chain, mv, kSlotOrient + 2 * t + 1);
            double R[3][3];
            rotationFromUniforms(a.x, a.y, b.x, R);
            double rsb[3];
            for (int r = 0; r < 3; ++r)
              rsb[r] = R[r][0] * c.offsets[sb][0] + R[r][1] * c.offsets[sb][1] + R[r][2] * c.offsets[sb][2];
            for (int i = 0; i < na; ++i)
              for (int r = 0; r < 3; ++r)
                sh.trial[t][i][r] = fb[r] - rsb[r] + R[r][0] * c.offsets[i][0] + R[r][1] * c.offsets[i][1] +
                                    R[r][2] * c.offsets[i][2];
          }
          __syncthreads();
          int others[kMaxAtoms];
          int no = 0;
          for (int i = 0; i < na; ++i)
            if (i != sb) others[no++] = i;
          for (int t = warp; t < p.k2; t += kWarps)
          {
            // gather the non-starting-bead atoms of trial t
            double op[kMaxAtoms][3];
            for (int j = 0; j < no; ++j)
              for (int d = 0; d < 3; ++d) op[j][d] = sh.trial[t][others[j]][d];
            int ov = 0;
            const double e = no > 0 ? warpExternal<QUINTIC>(p, chain, n, op, others, no, skip, &ov) : 0.0;
            if (lane == 0)
            {
              sh.setE[t] = e;
              sh.setOv[t] = ov;
            }
          }
          __syncthreads();
          if (threadIdx.x == 0)
          {
            double W2;
            int sel = selectTrial(sh.setE, sh.setOv, nullptr, p.k2, p.beta, uSel.y, &W2);
            if (retrace) sel = sh.setOv[0] ? -1 : 0;
            sh.ints[1] = sel;
            sh.dbl[5] = W2;
            sh.dbl[6] = sel >= 0 ? sh.setE[sel] : 0.0;
            if (sel >= 0)
              for (int i = 0; i < na; ++i)
                for (int d = 0; d < 3; ++d)
                {
                  if (insert)
                    sh.newPos[i][d] = sh.trial[sel][i][d];
                  else
                    sh.oldPos[i][d] = sh.trial[sel][i][d];
                }
          }
          __syncthreads();
          const int sel2 = sh.ints[1];
          if (sel2 >= 0)
          {
            const double W = W1 * sh.dbl[5];
            const double eExt = e1 + sh.dbl[6];
            double dEw = 0.0;
            if (p.use_ewald)
            {
              dEw = insert ? blockEwaldDelta(p, chain, sh.newPos, na, sh.oldPos, 0, tab, sh.red)
                           : blockEwaldDelta(p, chain, sh.newPos, 0, sh.oldPos, na, tab, sh.red);
              dEw += insert ? c.self_excl : -c.self_excl;
            }
            double pacc;
            if (insert)
              pacc = W < 1e-150 ? 0.0
                                : exp(-p.beta * dEw) * p.beta * p.fugacity * p.volume / static_cast<double>(n + 1) * W;
            else
              pacc = exp(-p.beta * dEw) * static_cast<double>(n) / (p.beta * p.fugacity * p.volume) / W;
            accepted = uChange.y < pacc;
            if (accepted)
            {
              if (insert)
              {
                if (threadIdx.x < na)
                  cpos[n * na + threadIdx.x] = make_double4(sh.newPos[threadIdx.x][0], sh.newPos[threadIdx.x][1],
                                                            sh.newPos[threadIdx.x][2], 0.0);
              }
              else if (m != n - 1 && threadIdx.x < na)
              {
                cpos[m * na + threadIdx.x] = cpos[(n - 1) * na + threadIdx.x];
              }
              if (p.use_ewald) blockAcceptEwald(p, chain);
              if (threadIdx.x == 0)
              {
                p.energy[chain] += insert ? (eExt + dEw) : (-eExt + dEw);
                p.n[chain] = insert ? n + 1 : n - 1;
              }
            }
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && record)
    {
      const int nn = p.n[chain];
      st[kind] += 1.0;
      st[4 + kind] += accepted ? 1.0 : 0.0;
      st[8] += nn;
      st[9] += static_cast<double>(nn) * nn;
      st[10] += p.energy[chain];
      st[11] += 1.0;
      const long long b = block_len > 0 ? static_cast<long long>(st[11] - 1.0) / block_len : 0;
      if (b < 5) st[12 + b] += nn;
    }
    __syncthreads();
  }
}
}  // namespace

struct rg_gcmc
{
  rg_ctx* ctx = nullptr;
  Params p{};
  int n_chains = 0;
  long long moves_done = 0;
  long long recorded = 0;
  long long block_len = 0;
  size_t shmem = 0;
  int max_moves_per_launch = 2048;
};

extern "C"
{
rg_status rg_gcmc_create(rg_system* system, rg_ewald* ewald, const rg_gcmc_component* comp,
                         const rg_gcmc_params* params, int n_chains, rg_gcmc** out)
{
  if (!system || !comp || !params || !out || n_chains < 1) return RG_ERR_INVALID_ARGUMENT;
  if (comp->n_atoms < 1 || comp->n_atoms > kMaxAtoms || comp->starting_bead < 0 || comp->starting_bead >= comp->n_atoms)
    return RG_ERR_INVALID_ARGUMENT;
  if (params->n_first_bead_trials < 1 || params->n_first_bead_trials > kMaxTrials ||
      params->n_orientation_trials < 1 || params->n_orientation_trials > kMaxTrials || params->max_molecules < 1)
    return RG_ERR_INVALID_ARGUMENT;
  rgd::FF ff;
  rgd::Box box;
  const double* grids[64];
  const double* ewald_grid = nullptr;
  int n_types, gdims[3];
  double gic[3][3];
  rg_ctx* ctx;
  rg_status st = rgd::systemExport(system, &ff, &box, grids, &ewald_grid, &n_types, gdims, gic, &ctx);
  if (st) return st;
  for (int i = 0; i < comp->n_atoms; ++i)
    if (comp->types[i] < 0 || comp->types[i] >= n_types) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_gcmc: type");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_gcmc* g = new rg_gcmc();
  g->ctx = ctx;
  g->n_chains = n_chains;
  Params& p = g->p;
  p.ff = ff;
  p.box = box;
  p.grid.nx = gdims[0];
  p.grid.ny = gdims[1];
  p.grid.nz = gdims[2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) p.grid.ic[a][b] = gic[a][b];
  p.comp.n_atoms = comp->n_atoms;
  p.comp.starting_bead = comp->starting_bead;
  for (int i = 0; i < comp->n_atoms; ++i)
  {
    p.comp.types[i] = comp->types[i];
    p.comp.charges[i] = comp->charges[i];
    p.comp.masses[i] = comp->masses[i];
    for (int d = 0; d < 3; ++d) p.comp.offsets[i][d] = comp->offsets[3 * i + d];
    p.vdw_grid[i] = comp->types[i] < 64 ? grids[comp->types[i]] : nullptr;
  }
  p.ewald_grid = ewald_grid;
  p.quintic = rgd::systemScheme(system) == RG_SCHEME_TRIQUINTIC ? 1 : 0;
  p.rcv_fw2 = params->cutoff_framework_vdw * params->cutoff_framework_vdw;
  p.rcv_mol2 = params->cutoff_molecule_vdw * params->cutoff_molecule_vdw;
  p.rcc2 = params->cutoff_coulomb * params->cutoff_coulomb;
  p.beta = params->beta;
  p.fugacity = params->fugacity;
  p.volume = box.volume;
  p.max_translation = params->max_translation;
  p.max_rotation = params->max_rotation;
  p.p_translation = params->p_translation;
  p.p_rotation = params->p_rotation;
  p.p_swap = params->p_swap;
  p.k1 = params->n_first_bead_trials;
  p.k2 = params->n_orientation_trials;
  p.capacity = params->max_molecules;
  p.seed = params->seed;
  p.use_ewald = (ewald != nullptr && ff.use_charge) ? 1 : 0;
  int64_t nk = 0;
  if (p.use_ewald)
  {
    const double2* s_rigid;
    double alpha, single_ion;
    st = rgd::ewaldExport(ewald, &p.kvec, &p.temp, &s_rigid, &nk, p.kmax, &alpha, &single_ion);
    if (st)
    {
      delete g;
      return st;
    }
    if (p.kmax[0] + 1 > kMaxK || p.kmax[1] + 1 > kMaxK || p.kmax[2] + 1 > kMaxK)
    {
      delete g;
      return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_gcmc: kmax per axis at most 15");
    }
    // self + exclusion energy added by one inserted molecule (ewald.cpp:1164-1238, new-atom terms, scaling 1)
    const double C = rg::coulombFactor();
    double se = 0.0;
    const double pself = C * alpha / std::sqrt(rg::kPi);
    for (int i = 0; i < comp->n_atoms; ++i) se -= pself * comp->charges[i] * comp->charges[i];
    for (int i = 0; i < comp->n_atoms; ++i)
      for (int j = i + 1; j < comp->n_atoms; ++j)
      {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d)
        {
          const double dd = comp->offsets[3 * i + d] - comp->offsets[3 * j + d];
          d2 += dd * dd;
        }
        const double r = std::sqrt(d2);
        se -= C * comp->charges[i] * comp->charges[j] * std::erf(alpha * r) / r;
      }
    p.comp.self_excl = se;
    p.nk = nk;
    // all chains start from the framework structure factor
    const size_t skb = sizeof(double2) * static_cast<size_t>(nk) * n_chains;
    cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&p.sk), skb);
    if (!err) err = cudaMalloc(reinterpret_cast<void**>(&p.dsk), skb);
    for (int c = 0; c < n_chains && !err; ++c)
      err = cudaMemcpyAsync(p.sk + static_cast<size_t>(c) * nk, s_rigid, sizeof(double2) * nk,
                            cudaMemcpyDeviceToDevice, ctx->stream);
    if (err)
    {
      rg_gcmc_destroy(g);
      return rg::cudaFail(ctx, err, "rg_gcmc_create (structure factors)");
    }
  }
  const size_t posb = sizeof(double4) * static_cast<size_t>(n_chains) * p.capacity * comp->n_atoms;
  cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&p.pos), posb);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&p.n), sizeof(int) * n_chains);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&p.energy), sizeof(double) * n_chains);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&p.stats), sizeof(double) * kStats * n_chains);
  if (!err) err = cudaMemsetAsync(p.pos, 0, posb, ctx->stream);
  if (!err) err = cudaMemsetAsync(p.n, 0, sizeof(int) * n_chains, ctx->stream);
  if (!err) err = cudaMemsetAsync(p.energy, 0, sizeof(double) * n_chains, ctx->stream);
  if (!err) err = cudaMemsetAsync(p.stats, 0, sizeof(double) * kStats * n_chains, ctx->stream);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (err)
  {
    rg_gcmc_destroy(g);
    return rg::cudaFail(ctx, err, "rg_gcmc_create");
  }
  const int stride = (p.kmax[0] + 1) + (p.kmax[1] + 1) + (p.kmax[2] + 1);
  g->shmem = sizeof(double2) * 2 * kMaxAtoms * (p.use_ewald ? stride : 1);
  *out = g;
  return RG_OK;
}

rg_status rg_gcmc_destroy(rg_gcmc* g)
{
  if (!g) return RG_OK;
  if (g->ctx) cudaStreamSynchronize(g->ctx->stream);
  cudaFree(g->p.pos);
  cudaFree(g->p.sk);
  cudaFree(g->p.dsk);
  cudaFree(g->p.n);
  cudaFree(g->p.energy);
  cudaFree(g->p.stats);
  delete g;
  return RG_OK;
}

rg_status rg_gcmc_run(rg_gcmc* g, int64_t moves, int record)
{
  if (!g || moves < 0) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = g->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (record && g->block_len == 0) g->block_len = moves / 5 > 0 ? moves / 5 : 1;
  int64_t left = moves;
  while (left > 0)
  {
    const int chunk = static_cast<int>(left < g->max_moves_per_launch ? left : g->max_moves_per_launch);
    if (g->p.quintic)
      gcmcKernel<true><<<g->n_chains, kThreads, g->shmem, ctx->stream>>>(g->p, g->moves_done, chunk, record,
                                                                         g->block_len);
    else
      gcmcKernel<false><<<g->n_chains, kThreads, g->shmem, ctx->stream>>>(g->p, g->moves_done, chunk, record,
                                                                          g->block_len);
    RG_CUDA(ctx, cudaGetLastError());
    g->moves_done += chunk;
    left -= chunk;
  }
  return RG_OK;
}

rg_status rg_gcmc_results(rg_gcmc* g, rg_gcmc_chain_result* out)
{
  if (!g || !out) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = g->ctx;
  std::vector<int> n(g->n_chains);
  std::vector<double> e(g->n_chains), s(static_cast<size_t>(kStats) * g->n_chains);
  RG_CUDA(ctx, cudaMemcpyAsync(n.data(), g->p.n, sizeof(int) * g->n_chains, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(e.data(), g->p.energy, sizeof(double) * g->n_chains, cudaMemcpyDeviceToHost,
                               ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(s.data(), g->p.stats, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < g->n_chains; ++c)
  {
    rg_gcmc_chain_result& r = out[c];
    std::memset(&r, 0, sizeof(r));
    const double* q = &s[static_cast<size_t>(c) * kStats];
    r.n_molecules = n[c];
    r.energy = e[c];
    for (int k = 0; k < 4; ++k)
    {
      r.attempted[k] = static_cast<int64_t>(q[k]);
      r.accepted[k] = static_cast<int64_t>(q[4 + k]);
    }
    r.sum_n = q[8];
    r.sum_n2 = q[9];
    r.sum_energy = q[10];
    r.samples = static_cast<int64_t>(q[11]);
    for (int b = 0; b < 5; ++b) r.block_n[b] = g->block_len > 0 ? q[12 + b] / static_cast<double>(g->block_len) : 0.0;
  }
  return RG_OK;
}

rg_status rg_gcmc_get_positions(rg_gcmc* g, int chain, double* xyz, int capacity_atoms, int* n_molecules)
{
  if (!g || !xyz || !n_molecules || chain < 0 || chain >= g->n_chains) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = g->ctx;
  int n = 0;
  RG_CUDA(ctx, cudaMemcpyAsync(&n, g->p.n + chain, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const int na = g->p.comp.n_atoms;
  if (n * na > capacity_atoms) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_gcmc_get_positions: buffer too small");
  std::vector<double4> pos(static_cast<size_t>(n) * na);
  if (n > 0)
    RG_CUDA(ctx, cudaMemcpyAsync(pos.data(), g->p.pos + static_cast<size_t>(chain) * g->p.capacity * na,
                                 sizeof(double4) * n * na, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n * na; ++i)
  {
    xyz[3 * i] = pos[i].x;
    xyz[3 * i + 1] = pos[i].y;
    xyz[3 * i + 2] = pos[i].z;
  }
  *n_molecules = n;
  return RG_OK;
}
}

extern "C" rg_status rg_gcmc_set_proposal(rg_gcmc* g, rg_proposal* proposal, const rg_box* unit_cell)
{
  if (!g) return RG_ERR_INVALID_ARGUMENT;
  Params& p = g->p;
  if (!proposal)
  {
    p.prop_cdf = nullptr;
    p.prop_q = nullptr;
    return RG_OK;
  }
  if (!unit_cell) return RG_ERR_INVALID_ARGUMENT;
  rg_status st = rgd::proposalExport(proposal, &p.prop_cdf, &p.prop_q, &p.prop_G, &p.prop_eps);
  if (st) return st;
  const rg::HostBox ub = rg::makeHostBox(unit_cell);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
    {
      p.uc[a][b] = ub.c[a][b];
      p.uic[a][b] = ub.ic[a][b];
    }
  // the simulation box must be an integer replication of the unit cell along each lattice vector
  for (int d = 0; d < 3; ++d)
  {
    double ratio = 0.0, n2 = 0.0;
    for (int r = 0; r < 3; ++r)
    {
      ratio += p.box.c[d][r] * ub.c[d][r];
      n2 += ub.c[d][r] * ub.c[d][r];
    }
    ratio /= n2;
    const int rep = static_cast<int>(std::lround(ratio));
    double err = 0.0;
    for (int r = 0; r < 3; ++r) err += std::fabs(p.box.c[d][r] - rep * ub.c[d][r]);
    if (rep < 1 || err > 1e-6)
    {
      p.prop_cdf = nullptr;
      p.prop_q = nullptr;
      return rg::fail(g->ctx, RG_ERR_INVALID_ARGUMENT, "rg_gcmc_set_proposal: box is not a replication of the unit cell");
    }
    p.rep[d] = rep;
  }
  return RG_OK;
}

// (b) Energies of CBMC / CFCMC trial positions and orientations on sm_100a.
//
// Replaces CBMC::computeExternalNonOverlappingEnergies (src/raspakit/cbmc/interactions.cpp:54-179) with its two
// callees CBMC::computeFrameworkMoleculeEnergy (cbmc/interactions_framework_molecule.cpp:31-104) and
// CBMC::computeInterMolecularEnergy (cbmc/interactions_intermolecular.cpp:22-95).
//
// A system (rg_system) keeps on the device: the pair table, the simulation box, the framework atoms, the tricubic
// grids (one per pseudo-atom type plus the unit-charge Ewald grid) and the adsorbate atoms. One launch evaluates all
// trials of a growth step: the grid is (trial, chunk), sized to one wave of resident CTAs; each CTA stages the trial's
// atoms in shared memory (a call of up to 32 trial atoms brings them in the launch parameters, so it costs one launch
// and one synchronisation), the threads of chunks 1.. stride over their chunk of partners (framework atoms for trial
// atoms without a grid, then adsorbate atoms from other molecules), and the per-trial totals are reduced in a fixed
// order by the last CTA of the trial. Trial atoms with a grid (and not fractional) take the grid branch in chunk 0:
// one tricubic interpolation of their VDW grid and, with charges, q times the unit-charge Ewald grid. A trial is flagged as overlapping if any VDW pair energy or
// interpolated VDW energy exceeds the overlap criterion, which is the reference's std::nullopt. Arithmetic: FP64 by
// default; with RG_PRECISION_FP32C (rg_system_set_precision) the Lennard-Jones pair terms are FP32 from the FP64
// minimum-image displacement and each thread sums them in TwoSum-compensated FP32 pairs, folded into the FP64 totals;
// the real-space Coulomb pairs and the grid branch stay FP64 (charged-framework terms cancel by orders of magnitude).
//
// The same kernel serves the other callers of these pair loops: a call of two trial sets of their own sizes and
// cutoffs (new and old atoms of a translation or rotation, Interactions::computeFrameworkMoleculeEnergyDifference
// and computeInterMolecularEnergyDifference, interactions/framework_molecule.cpp:117-252, intermolecular.cpp:198-290;
// full and inner cutoffs of CBMC::computeDualCutOffCorrection, cbmc/interactions.cpp:181-251), and the two per-trial
// tests of computeExternalNonOverlappingEnergies that run before the pair loops: CBMC::insideBlockedPockets
// (cbmc/interactions.cpp:25-52) and CBMC::computeExternalFieldEnergy (cbmc/interactions_external_field.cpp:22-200),
// both in the grid-branch chunk.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"
#include "fastmath.cuh"

namespace
{
constexpr int kThreads = 256;
constexpr int kMinChunk = 256;         // partner atoms per CTA at least (a call fills the GPU with smaller chunks)
constexpr int kMaxChunk = 4096;         // and at most
constexpr int kMaxTrialAtoms = 64;     // atoms of one trial set
constexpr int kNumOut = 13;            // fmVDW, fmCharge, mmVDW, mmCharge, dudl VDW[4], dudl charge[4], external field
constexpr int kParamTrialAtoms = 32;   // trial sets of up to this many atoms in total travel in the launch parameters
}  // namespace

struct rg_system
{
  rg_ctx* ctx = nullptr;
  int n_types = 0;
  rgd::FF ff{};
  rgd::Box box{};
  double overlap = 1e6;
  // device buffers
  double* tables = nullptr;   // eps4, sig2, shift (3*n*n) followed by lj as ints
  rg_atom* fw = nullptr;
  int n_fw = 0;
  rg_atom* mol = nullptr;
  int n_mol = 0;
  int mol_cap = 0;
  std::vector<double*> grids;   // n_types + 1 slots (last = unit-charge Ewald grid); owned device copies
  std::vector<int> grid_owned;
  int gnx = 0, gny = 0, gnz = 0;
  double gic[3][3]{};
  // per-launch scratch
  rg_atom* trials = nullptr;
  int trial_cap = 0;
  double* partial = nullptr;
  int partial_cap = 0;
  unsigned int* counters = nullptr;
  int counter_cap = 0;
  rg_trial_energy* out = nullptr;
  int out_cap = 0;
  rg_atom* trials_host = nullptr;     // pinned
  rg_trial_energy* out_host = nullptr;    // mapped pinned: the last CTA of each trial writes its result here directly
  rg_trial_energy* out_mapped = nullptr;  // device view of out_host
  int precision = RG_PRECISION_FP64;      // of rg_cbmc_external_energies
  int sms = 148;
  int resident[4] = {0, 0, 0, 0};         // CTAs per SM of trialEnergyKernel<F32, QUINTIC> (0 = not yet queried)
  int scheme = RG_SCHEME_TRICUBIC;        // values per grid point: 8 (tricubic) or 27 (triquintic)
  // the force field's cutoffs and flags read by the difference and dual-cutoff calls
  double rc_fw = 12.0, rc_mol = 12.0, rc_coul = 12.0;
  bool omit_inter = false;
  // blocked pockets of the component (Cartesian centre, radius) and the framework unit cell for their minimum image
  double4* pockets = nullptr;
  int n_pockets = 0;
  rgd::Box pocket_box{};
  // external field: surface type, geometry parameters and an optional grid over its own box
  bool ext_on = false;
  int ext_type = 0;
  double ext_geom[4] = {0, 0, 0, 0};
  double* ext_grid = nullptr;
  bool ext_grid_owned = false;
  int egnx = 0, egny = 0, egnz = 0;
  double egic[3][3]{};
};

namespace
{
struct TrialArgs
{
  rgd::FF ff;
  rgd::Box box;
  const rg_atom* fw;
  int n_fw;
  const rg_atom* mol;
  int n_mol;
  const rg_atom* trials;
  int atoms_per_trial;
  int skip;
  long long skip_background;
  double rcv_fw2, rcv_mol2, rcc2;
  const double* grid[64];  // per type, null = no grid (types >= 64 have none)
  const double* ewald_grid;
  int gnx, gny, gnz;
  double gic[3][3];
  int n_chunks;            // chunk 0: the grid branch; chunks 1..: partner atoms
  int chunk;               // partner atoms per CTA
  int fw_partners;         // framework atoms scanned (0 if every trial atom has a grid)
  double* partial;         // [trial][chunk][kNumOut + 1]
  unsigned int* counters;  // per trial
  rg_trial_energy* out;
  // two trial sets of counts[t] atoms (stored atoms_per_trial apart) with their own squared cutoffs (framework VDW,
  // molecule VDW, Coulomb); otherwise every set has atoms_per_trial atoms and the cutoffs above
  int paired;
  int counts[2];
  double cut2[2][3];
  // blocked pockets: Cartesian centre and radius, minimum image in pocket_box
  const double4* pockets;
  int n_pockets;
  rgd::Box pocket_box;
  // external field: ext_on, the surface type and its geometry, or a grid (ext_grid) over its own box
  int ext_on;
  int ext_type;
  double ext_geom[4];
  const double* ext_grid;
  int egnx, egny, egnz;
  double egic[3][3];
};

// the trial atoms of a small call, passed by value in the launch parameters (no copy before the launch)
struct TrialParam
{
  rg_atom a[kParamTrialAtoms];
};

// FP32 form of rgd::pairVDW: the same soft-core formula (pair_vdw.ixx:85-101) with the table entries rounded to FP32.
__device__ __forceinline__ float2 pairVDWf(const rgd::FF& ff, float sA, float sB, float rr, int tA, int tB)
{
  const int idx = tA * ff.n + tB;
  if (!ff.lj[idx]) return make_float2(0.0f, 0.0f);
  const float scaling = sA * sB;
  const float arg1 = static_cast<float>(ff.eps4[idx]);
  const float arg2 = static_cast<float>(ff.sig2[idx]);
  const float arg3 = static_cast<float>(ff.shift[idx]);
  const float temp = rr * rgd::rcpRn(arg2);
  const float temp3 = temp * temp * temp;
  const float inv_scaling = 1.0f - scaling;
  const float rri3 = rgd::rcpRn(temp3 + 0.5f * inv_scaling * inv_scaling);
  const float rri6 = rri3 * rri3;
  const float term = arg1 * (rri3 * (rri3 - 1.0f)) - arg3;
  const float dlambda_term = arg1 * scaling * inv_scaling * (2.0f * rri6 * rri3 - rri6);
  return make_float2(scaling * term, term + dlambda_term);
}

// FP32 sum with its rounding error carried exactly (Knuth TwoSum) in a second FP32 word
struct Sum32
{
  float hi = 0.0f, lo = 0.0f;
  __device__ __forceinline__ void add(float x)
  {
    const float t = hi + x;
    const float z = t - hi;
    lo += (hi - (t - z)) + (x - z);
    hi = t;
  }
  __device__ __forceinline__ double value() const { return static_cast<double>(hi) + static_cast<double>(lo); }
};

// acc[g - 1] += x for a dU/dlambda group g in 1..4, with constant indices so that the accumulators stay in registers
template <typename T, typename V>
__device__ __forceinline__ void addToGroup(T* acc, int g, V x)
{
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (g == k + 1) acc[k] += x;
}

__device__ __forceinline__ Sum32& operator+=(Sum32& s, float x)
{
  s.add(x);
  return s;
}

// CBMC::computeExternalFieldEnergy for one atom (cbmc/interactions_external_field.cpp:22-200): a grid, scaled by the
// atom's VDW scaling, takes precedence; otherwise the Muller-Brown surface, the x y z test function, or a cylinder or
// rectangle along a cell axis whose outside is forbidden (returns false: the reference's std::nullopt); every other
// surface type adds nothing. Positions are used as given, unwrapped, as in the reference.
template <bool QUINTIC>
__device__ bool externalFieldEnergy(const TrialArgs& a, const rg_atom& A, double* e)
{
  *e = 0.0;
  if (a.ext_grid)
  {
    rgd::Grid g{a.ext_grid, a.egnx, a.egny, a.egnz, {}};
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) g.ic[r][c] = a.egic[r][c];
    *e = A.scaling_vdw * (QUINTIC ? rgd::interpolateQuintic(g, A.x, A.y, A.z, nullptr) : rgd::interpolate(g, A.x, A.y, A.z));
    return true;
  }
  const int type = a.ext_type;
  if (type == 8)  // MullerBrown
  {
    const double Ak[4] = {-200.0, -100.0, -170.0, -15.0}, ak[4] = {-1.0, -1.0, -6.5, -0.7},
                 x0[4] = {1.0, 0.0, -0.5, -1.0}, bk[4] = {0.0, 0.0, 11.0, 0.6}, y0[4] = {0.0, 0.5, 1.5, 1.0},
                 ck[4] = {-10.0, -10.0, -6.5, 0.7};
    double sum = 0.0;
    for (int i = 0; i < 4; ++i)
      sum += Ak[i] * exp(ak[i] * (A.x - x0[i]) * (A.x - x0[i]) + bk[i] * (A.x - x0[i]) * (A.y - y0[i]) +
                         ck[i] * (A.y - y0[i]) * (A.y - y0[i]));
    *e = sum;
    return true;
  }
  if (type == 3)  // ThirdOrderPolynomialTestFunction
  {
    *e = A.x * A.y * A.z;
    return true;
  }
  if (type >= 11 && type <= 16)  // CylinderX/Y/Z, RectangleX/Y/Z: the line through the box centre along one axis
  {
    const int axis = (type - 11) % 3;
    double fb[3] = {0.5, 0.5, 0.5}, fe[3] = {0.5, 0.5, 0.5};
    fb[axis] = 0.0;
    fe[axis] = 1.0;
    double cb[3], ce[3];
    for (int r = 0; r < 3; ++r)
    {
      cb[r] = a.box.c[0][r] * fb[0] + a.box.c[1][r] * fb[1] + a.box.c[2][r] * fb[2];
      ce[r] = a.box.c[0][r] * fe[0] + a.box.c[1][r] * fe[1] + a.box.c[2][r] * fe[2];
    }
    double v[3] = {ce[0] - cb[0], ce[1] - cb[1], ce[2] - cb[2]};
    const double len = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int r = 0; r < 3; ++r) v[r] /= len;
    const double d[3] = {A.x - cb[0], A.y - cb[1], A.z - cb[2]};
    const double w[3] = {d[1] * v[2] - d[2] * v[1], d[2] * v[0] - d[0] * v[2], d[0] * v[1] - d[1] * v[0]};
    if (type <= 13) return w[0] * w[0] + w[1] * w[1] + w[2] * w[2] < a.ext_geom[0] * a.ext_geom[0];
    if (type == 14) return fabs(w[1]) < a.ext_geom[0] && fabs(w[2]) < a.ext_geom[1];
    if (type == 15) return fabs(w[2]) < a.ext_geom[0] && fabs(w[0]) < a.ext_geom[1];
    return fabs(w[1]) < a.ext_geom[0] && fabs(w[0]) < a.ext_geom[1];
  }
  return true;
}

template <bool F32, bool QUINTIC>
__global__ void __launch_bounds__(kThreads) trialEnergyKernel(TrialArgs a, TrialParam small)
{
  const int trial = blockIdx.x;
  const int chunk = blockIdx.y;
  __shared__ rg_atom sT[kMaxTrialAtoms];
  __shared__ int sGridBranch[kMaxTrialAtoms];
  __shared__ double red[kThreads / 32][kNumOut + 1];
  __shared__ bool last;
  const int stride = a.atoms_per_trial;
  const int nA = a.paired ? a.counts[trial] : stride;
  const double rcv_fw2 = a.paired ? a.cut2[trial][0] : a.rcv_fw2;
  const double rcv_mol2 = a.paired ? a.cut2[trial][1] : a.rcv_mol2;
  const double rcc2 = a.paired ? a.cut2[trial][2] : a.rcc2;
  for (int i = threadIdx.x; i < nA; i += blockDim.x)
  {
    sT[i] = a.trials ? a.trials[static_cast<long long>(trial) * stride + i] : small.a[trial * stride + i];
    const int t = sT[i].type;
    sGridBranch[i] = (t < 64 && a.grid[t] != nullptr && !rgd::fractionalOf(sT[i])) ? 1 : 0;
  }
  __syncthreads();

  double acc[kNumOut];
#pragma unroll
  for (int c = 0; c < kNumOut; ++c) acc[c] = 0.0;
  Sum32 acc32[F32 ? 12 : 1];  // the pair terms (the external field stays FP64)
  double overlap = 0.0;

  // chunk 0 is the grid branch alone: one thread per (trial atom, grid), the VDW grid on even threads and q times the
  // unit-charge Ewald grid on odd ones, so that no partner chunk waits for an interpolation
  if (chunk == 0)
  {
    for (int j = threadIdx.x; j < 2 * nA; j += blockDim.x)
    {
      const int i = j >> 1;
      if (i == a.skip || !sGridBranch[i]) continue;
      const bool ewald = (j & 1) != 0;
      if (ewald && !(a.ff.use_charge && a.ewald_grid)) continue;
      rgd::Grid g{ewald ? a.ewald_grid : a.grid[sT[i].type], a.gnx, a.gny, a.gnz, {}};
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) g.ic[r][c] = a.gic[r][c];
      const double e = QUINTIC ? rgd::interpolateQuintic(g, sT[i].x, sT[i].y, sT[i].z, nullptr)
                               : rgd::interpolate(g, sT[i].x, sT[i].y, sT[i].z);
      if (ewald)
        acc[1] += sT[i].charge * e;
      else
      {
        if (e > a.ff.overlap) overlap = fmax(overlap, 1.0);
        acc[0] += e;
      }
    }
    // blocked pockets: every atom of the set, the skipped one included (insideBlockedPockets tests the whole set);
    // a hit marks the trial 2 (dropped)
    for (int j = threadIdx.x; j < nA * a.n_pockets; j += blockDim.x)
    {
      const int i = j / a.n_pockets;
      const double4 pk = a.pockets[j - i * a.n_pockets];
      double dx = sT[i].x - pk.x, dy = sT[i].y - pk.y, dz = sT[i].z - pk.z;
      rgd::pbc(a.pocket_box, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz < sT[i].scaling_vdw * (pk.w * pk.w)) overlap = fmax(overlap, 2.0);
    }
    if (a.ext_on)
      for (int i = threadIdx.x; i < nA; i += blockDim.x)
      {
        if (i == a.skip) continue;
        double e;
        if (!externalFieldEnergy<QUINTIC>(a, sT[i], &e)) overlap = fmax(overlap, 1.0);
        acc[12] += e;
      }
  }

  const long long total = static_cast<long long>(a.fw_partners) + a.n_mol;
  const long long begin = chunk == 0 ? total : static_cast<long long>(chunk - 1) * a.chunk;
  const long long end = begin + a.chunk < total ? begin + a.chunk : total;
  for (long long p = begin + threadIdx.x; p < end; p += blockDim.x)
  {
    const bool isFw = p < a.fw_partners;
    const rg_atom B = isFw ? a.fw[p] : a.mol[p - a.fw_partners];
    if (!isFw && a.skip_background >= 0 && static_cast<long long>(B.molecule_id) == a.skip_background) continue;
    const int gB = rgd::groupOf(B);
    for (int i = 0; i < nA; ++i)
    {
      if (i == a.skip) continue;
      const rg_atom& A = sT[i];
      if (isFw && sGridBranch[i]) continue;
      if (!isFw && A.molecule_id == B.molecule_id) continue;
      // dr = partner - trial in both loops (interactions_framework_molecule.cpp:86-88,
      // interactions_intermolecular.cpp:66-68)
      double dx = B.x - A.x, dy = B.y - A.y, dz = B.z - A.z;
      rgd::pbc(a.box, dx, dy, dz);
      const double rr = dx * dx + dy * dy + dz * dz;
      const double rcv2 = isFw ? rcv_fw2 : rcv_mol2;
      const int gA = rgd::groupOf(A);
      if constexpr (F32)
      {
        const float rrf = static_cast<float>(rr);
        if (rr < rcv2)
        {
          const float2 f = pairVDWf(a.ff, static_cast<float>(B.scaling_vdw), static_cast<float>(A.scaling_vdw), rrf,
                                    B.type, A.type);
          if (static_cast<double>(f.x) > a.ff.overlap) overlap = fmax(overlap, 1.0);
          if (isFw)
            acc32[0].add(f.x);
          else
            acc32[2].add(f.x);
          addToGroup(acc32 + 4, gB, static_cast<float>(A.scaling_vdw) * f.y);
          addToGroup(acc32 + 4, gA, static_cast<float>(B.scaling_vdw) * f.y);
        }
        if (a.ff.use_charge && rr < rcc2)
        {
          // the real-space Coulomb pair stays FP64: the +2.05 / -1.025 e framework terms (up to ~1e5 K each) cancel
          // to a few 1e2 K, and FP32 rounding of them alone exceeds 1e-6 of a trial's energy
          const double2 f = rgd::pairCoulomb(a.ff, B.scaling_coulomb, A.scaling_coulomb, sqrt(rr), B.charge, A.charge);
          if (isFw)
            acc[1] += f.x;
          else
            acc[3] += f.x;
          addToGroup(acc + 8, gB, A.scaling_coulomb * f.y);
          addToGroup(acc + 8, gA, B.scaling_coulomb * f.y);
        }
      }
      else
      {
        if (rr < rcv2)
        {
          const double2 f = rgd::pairVDW(a.ff, B.scaling_vdw, A.scaling_vdw, rr, B.type, A.type);
          if (f.x > a.ff.overlap) overlap = fmax(overlap, 1.0);
          if (isFw)
            acc[0] += f.x;
          else
            acc[2] += f.x;
          // addDudlambdaVDW(groupIdA(partner), groupIdB(trial), ...) (running_energy.ixx:258-263)
          addToGroup(acc + 4, gB, A.scaling_vdw * f.y);
          addToGroup(acc + 4, gA, B.scaling_vdw * f.y);
        }
        if (a.ff.use_charge && rr < rcc2)
        {
          const double r = sqrt(rr);
          const double2 f = rgd::pairCoulomb(a.ff, B.scaling_coulomb, A.scaling_coulomb, r, B.charge, A.charge);
          if (isFw)
            acc[1] += f.x;
          else
            acc[3] += f.x;
          addToGroup(acc + 8, gB, A.scaling_coulomb * f.y);
          addToGroup(acc + 8, gA, B.scaling_coulomb * f.y);
        }
      }
    }
  }

  if constexpr (F32)
  {
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] += acc32[c].value();
  }
  // block reduction (fixed order), then the last CTA of this trial sums the chunks in order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c <= kNumOut; ++c)
  {
    double x = c < kNumOut ? acc[c] : overlap;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = (c < kNumOut) ? x + y : fmax(x, y);
    }
    if (lane == 0) red[warp][c] = x;
  }
  __syncthreads();
  // one thread per channel: the CTA's partial over the warps, then (last CTA) the trial's total over the chunks
  const int c = threadIdx.x;
  if (c <= kNumOut)
  {
    double x = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) x = (c < kNumOut) ? x + red[w][c] : fmax(x, red[w][c]);
    a.partial[(static_cast<long long>(trial) * a.n_chunks + chunk) * (kNumOut + 1) + c] = x;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    const unsigned int done = atomicAdd(a.counters + trial, 1u);
    last = (done == static_cast<unsigned int>(a.n_chunks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the trial's total over its chunks: 16 threads per channel sum the chunks j, j + 16, ... (their loads in flight
  // together), then each channel's 16 sub-sums in order
  static_assert(kThreads == 16 * 16 && kNumOut + 1 <= 16, "16 threads for each of at most 16 channels");
  __shared__ double sub[kNumOut + 1][16];
  __shared__ double tot[kNumOut + 1];
  const int cc = threadIdx.x >> 4, j0 = threadIdx.x & 15;
  if (cc <= kNumOut)
  {
    const double* src = a.partial + static_cast<long long>(trial) * a.n_chunks * (kNumOut + 1) + cc;
    double x = 0.0;
#pragma unroll 4
    for (int ch = j0; ch < a.n_chunks; ch += 16)
    {
      const double y = __ldcg(src + static_cast<long long>(ch) * (kNumOut + 1));
      x = (cc < kNumOut) ? x + y : fmax(x, y);
    }
    sub[cc][j0] = x;
  }
  __syncthreads();
  if (c <= kNumOut)
  {
    double x = 0.0;
    for (int j = 0; j < 16; ++j) x = (c < kNumOut) ? x + sub[c][j] : fmax(x, sub[c][j]);
    tot[c] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    rg_trial_energy o;
    o.framework_vdw = tot[0];
    o.framework_charge = tot[1];
    o.molecule_vdw = tot[2];
    o.molecule_charge = tot[3];
    for (int g = 0; g < 4; ++g)
    {
      o.dudlambda_vdw[g] = tot[4 + g];
      o.dudlambda_charge[g] = tot[8 + g];
    }
    o.external_field_vdw = tot[12];
    o.overlap = static_cast<int32_t>(tot[kNumOut]);  // 0, 1 (overlap) or 2 (blocked pocket)
    o.pad = 0;
    a.out[trial] = o;
    a.counters[trial] = 0u;
  }
}

template <typename T>
rg_status growDevice(rg_ctx* ctx, T** p, int* cap, int need)
{
  if (*cap >= need && *p) return RG_OK;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (*p) RG_CUDA(ctx, cudaFree(*p));
  *p = nullptr;
  int grow = need + need / 2 + 16;
  RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * static_cast<size_t>(grow)));
  *cap = grow;
  return RG_OK;
}
}  // namespace

extern "C"
{
rg_status rg_system_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* box, const rg_atom* framework_atoms,
                           int n_framework_atoms, rg_system** out)
{
  if (!ctx || !ff || !box || !out || n_framework_atoms < 0 || (n_framework_atoms > 0 && !framework_atoms))
    return RG_ERR_INVALID_ARGUMENT;
  if (rg_status fs = rg::checkFinite(ctx, framework_atoms, n_framework_atoms, "rg_system_create")) return fs;
  if (rg_status fs = rg::checkFiniteBox(ctx, box, "rg_system_create")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_system* s = new rg_system();
  s->ctx = ctx;
  const int n = ff->n_types;
  s->n_types = n;
  std::vector<double> tab(3 * n * n);
  std::vector<int> lj(n * n);
  for (int i = 0; i < n * n; ++i)
  {
    tab[i] = 4.0 * ff->epsilon[i];
    tab[n * n + i] = ff->sigma[i] * ff->sigma[i];
    tab[2 * n * n + i] = ff->shift[i];
    lj[i] = ff->lj[i];
  }
  // all copies on the context stream, synchronised before returning (the legacy default stream does not order with it)
  cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&s->tables), sizeof(double) * 3 * n * n + sizeof(int) * n * n);
  if (!err)
    err = cudaMemcpyAsync(s->tables, tab.data(), sizeof(double) * 3 * n * n, cudaMemcpyHostToDevice, ctx->stream);
  if (!err)
    err = cudaMemcpyAsync(s->tables + 3 * n * n, lj.data(), sizeof(int) * n * n, cudaMemcpyHostToDevice, ctx->stream);
  if (!err && n_framework_atoms > 0)
  {
    err = cudaMalloc(reinterpret_cast<void**>(&s->fw), sizeof(rg_atom) * n_framework_atoms);
    if (!err)
      err = cudaMemcpyAsync(s->fw, framework_atoms, sizeof(rg_atom) * n_framework_atoms, cudaMemcpyHostToDevice,
                            ctx->stream);
  }
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (!err) err = cudaMallocHost(reinterpret_cast<void**>(&s->trials_host), sizeof(rg_atom) * 4096);
  if (!err)
    err = cudaHostAlloc(reinterpret_cast<void**>(&s->out_host), sizeof(rg_trial_energy) * 4096, cudaHostAllocMapped);
  if (!err) err = cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->out_mapped), s->out_host, 0);
  if (!err) err = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (err)
  {
    rg_status st = rg::cudaFail(ctx, err, "rg_system_create");
    rg_system_destroy(s);
    return st;
  }
  s->n_fw = n_framework_atoms;
  s->ff.n = n;
  s->ff.eps4 = s->tables;
  s->ff.sig2 = s->tables + n * n;
  s->ff.shift = s->tables + 2 * n * n;
  s->ff.lj = reinterpret_cast<const int*>(s->tables + 3 * n * n);
  s->ff.alpha = ff->ewald_alpha;
  s->ff.coul = rg::coulombFactor();
  s->ff.overlap = ff->overlap_criteria;
  s->ff.use_charge = ff->use_charge;
  s->rc_fw = ff->cutoff_framework_vdw;
  s->rc_mol = ff->cutoff_molecule_vdw;
  s->rc_coul = ff->cutoff_coulomb;
  s->omit_inter = ff->omit_inter != 0;
  rg::HostBox hb = rg::makeHostBox(box);
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
    {
      s->box.c[c][r] = hb.c[c][r];
      s->box.ic[c][r] = hb.ic[c][r];
    }
  s->box.triclinic = hb.triclinic ? 1 : 0;
  s->box.volume = hb.volume;
  s->grids.assign(n + 1, nullptr);
  s->grid_owned.assign(n + 1, 0);
  *out = s;
  return RG_OK;
}

rg_status rg_system_destroy(rg_system* s)
{
  if (!s) return RG_OK;
  if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
  cudaFree(s->tables);
  cudaFree(s->fw);
  cudaFree(s->mol);
  for (size_t i = 0; i < s->grids.size(); ++i)
    if (s->grid_owned[i]) cudaFree(s->grids[i]);
  cudaFree(s->trials);
  cudaFree(s->partial);
  cudaFree(s->counters);
  cudaFree(s->out);
  cudaFree(s->pockets);
  if (s->ext_grid_owned) cudaFree(s->ext_grid);
  if (s->trials_host) cudaFreeHost(s->trials_host);
  if (s->out_host) cudaFreeHost(s->out_host);
  delete s;
  return RG_OK;
}

rg_status rg_system_set_grid(rg_system* s, int index, const rg_box* unit_cell, int nx, int ny, int nz,
                             const double* data, int data_on_device)
{
  if (!s || !unit_cell || !data || index < 0 || index > s->n_types || nx < 2 || ny < 2 || nz < 2)
    return RG_ERR_INVALID_ARGUMENT;
  if (index < s->n_types && index >= 64)
    return rg::fail(s->ctx, RG_ERR_UNSUPPORTED, "rg_system_set_grid: grids only for pseudo-atom types < 64");
  rg_ctx* ctx = s->ctx;
  bool first = true;
  for (int i = 0; i <= s->n_types; ++i)
    if (s->grids[i]) first = false;
  if (!first && (nx != s->gnx || ny != s->gny || nz != s->gnz))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_set_grid: all grids of a system share one shape");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(double) * s->scheme * static_cast<size_t>(nx) * ny * nz;
  if (s->grid_owned[index]) RG_CUDA(ctx, cudaFree(s->grids[index]));
  s->grids[index] = nullptr;
  s->grid_owned[index] = 0;
  if (data_on_device)
  {
    s->grids[index] = const_cast<double*>(data);  // borrowed: the caller keeps it alive
  }
  else
  {
    RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&s->grids[index]), bytes));
    s->grid_owned[index] = 1;
    RG_CUDA(ctx, cudaMemcpyAsync(s->grids[index], data, bytes, cudaMemcpyHostToDevice, ctx->stream));
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  rg::HostBox hb = rg::makeHostBox(unit_cell);
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) s->gic[c][r] = hb.ic[c][r];
  s->gnx = nx;
  s->gny = ny;
  s->gnz = nz;
  return RG_OK;
}

rg_status rg_system_set_molecules(rg_system* s, const rg_atom* atoms, int n)
{
  if (!s || n < 0 || (n > 0 && !atoms)) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = s->ctx;
  if (rg_status fs = rg::checkFinite(ctx, atoms, n, "rg_system_set_molecules")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_status st = growDevice(ctx, &s->mol, &s->mol_cap, n > 0 ? n : 1);
  if (st) return st;
  if (n > 0) RG_CUDA(ctx, cudaMemcpyAsync(s->mol, atoms, sizeof(rg_atom) * n, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the caller's atom buffer is pageable
  s->n_mol = n;
  return RG_OK;
}

rg_status rg_system_set_precision(rg_system* s, int precision)
{
  if (!s || (precision != RG_PRECISION_FP64 && precision != RG_PRECISION_FP32C)) return RG_ERR_INVALID_ARGUMENT;
  s->precision = precision;
  return RG_OK;
}

rg_status rg_system_set_interpolation_scheme(rg_system* s, int scheme)
{
  if (!s) return RG_ERR_INVALID_ARGUMENT;
  if (scheme != RG_SCHEME_TRICUBIC && scheme != RG_SCHEME_TRIQUINTIC)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_set_interpolation_scheme: RG_SCHEME_TRICUBIC or "
                                                     "RG_SCHEME_TRIQUINTIC");
  for (int i = 0; i <= s->n_types; ++i)
    if (s->grids[i] && scheme != s->scheme)
      return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT,
                      "rg_system_set_interpolation_scheme: set the scheme before the first grid");
  s->scheme = scheme;
  return RG_OK;
}

}  // extern "C"

namespace
{
// What one launch of trialEnergyKernel evaluates.
struct TrialCall
{
  const rg_atom* trials = nullptr;  // n_trials sets, atoms_per_trial apart
  int n_trials = 0;
  int atoms_per_trial = 1;
  int skip = -1;
  long long skip_background = -1;
  double cut[3] = {12.0, 12.0, 12.0};  // framework VDW, molecule VDW, Coulomb
  bool paired = false;                 // two sets of counts[0] and counts[1] atoms, cutoffs cut_pair[t]
  int counts[2] = {0, 0};
  double cut_pair[2][3] = {};
  bool framework = true;               // framework partners (and the grid branch)
  bool molecules = true;               // adsorbate partners
  bool grids = true;                   // the grid branch for atoms with a grid; false: pair loop for every atom
  bool pockets_and_field = true;       // blocked pockets and the external field
  const char* what = "rg_cbmc_external_energies";
};

rg_status runTrials(rg_system* s, const TrialCall& c, rg_trial_energy* out)
{
  rg_ctx* ctx = s->ctx;
  const int n_trials = c.n_trials, atoms_per_trial = c.atoms_per_trial;
  if (n_trials == 0) return RG_OK;
  const int nt_atoms = n_trials * atoms_per_trial;
  if (rg_status fs = rg::checkFinite(ctx, c.trials, nt_atoms, c.what)) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  auto hasGrid = [&](const rg_atom& at)
  {
    const int t = at.type;
    return c.grids && t < 64 && t < s->n_types && s->grids[t] && !((at.group_fractional >> 4) != 0);
  };
  // does any trial atom need the framework pair loop?
  bool needFw = false;
  for (int tr = 0; tr < n_trials && !needFw && c.framework; ++tr)
  {
    const int n = c.paired ? c.counts[tr] : atoms_per_trial;
    for (int i = 0; i < n && !needFw; ++i)
    {
      if (i == c.skip) continue;
      if (!hasGrid(c.trials[tr * atoms_per_trial + i])) needFw = true;
    }
  }
  const int fw_partners = needFw ? s->n_fw : 0;
  const int n_mol = c.molecules ? s->n_mol : 0;
  const long long total = static_cast<long long>(fw_partners) + n_mol;
  const bool f32 = s->precision == RG_PRECISION_FP32C;
  const bool quintic = s->scheme == RG_SCHEME_TRIQUINTIC;
  const auto kernel = f32 ? (quintic ? trialEnergyKernel<true, true> : trialEnergyKernel<true, false>)
                          : (quintic ? trialEnergyKernel<false, true> : trialEnergyKernel<false, false>);
  int& resident = s->resident[(f32 ? 1 : 0) + (quintic ? 2 : 0)];
  if (resident == 0)
  {
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kThreads, 0);
    if (err) return rg::cudaFail(ctx, err, "rg_cbmc_external_energies: occupancy");
    resident = std::max(1, resident);
  }
  // chunks of partners: as many CTAs as are resident at once (one wave, the grid-branch chunk included), each with
  // at least kMinChunk and at most kMaxChunk partners
  const long long want = std::max<long long>(1, static_cast<long long>(resident) * s->sms / n_trials - 1);
  long long chunk = total > 0 ? (total + want - 1) / want : 1;
  chunk = std::min<long long>(kMaxChunk, std::max<long long>(kMinChunk, chunk));
  const int n_chunks = 1 + static_cast<int>(total > 0 ? (total + chunk - 1) / chunk : 0);
  rg_status st = RG_OK;
  const bool inParams = nt_atoms <= kParamTrialAtoms;
  if (!inParams) st = growDevice(ctx, &s->trials, &s->trial_cap, nt_atoms);
  if (!st) st = growDevice(ctx, &s->partial, &s->partial_cap, n_trials * n_chunks * (kNumOut + 1));
  if (!st && s->counter_cap < n_trials)
  {
    st = growDevice(ctx, &s->counters, &s->counter_cap, n_trials);
    if (!st) RG_CUDA(ctx, cudaMemsetAsync(s->counters, 0, sizeof(unsigned int) * s->counter_cap, ctx->stream));
  }
  if (st) return st;
  TrialParam small{};
  if (inParams)
    std::memcpy(small.a, c.trials, sizeof(rg_atom) * nt_atoms);
  else
  {
    // the pinned staging buffer is free: every call ends by synchronising the stream
    std::memcpy(s->trials_host, c.trials, sizeof(rg_atom) * nt_atoms);
    RG_CUDA(ctx, cudaMemcpyAsync(s->trials, s->trials_host, sizeof(rg_atom) * nt_atoms, cudaMemcpyHostToDevice,
                                 ctx->stream));
  }
  TrialArgs a{};
  a.ff = s->ff;
  a.box = s->box;
  a.fw = s->fw;
  a.n_fw = s->n_fw;
  a.mol = s->mol;
  a.n_mol = n_mol;
  a.trials = inParams ? nullptr : s->trials;
  a.atoms_per_trial = atoms_per_trial;
  a.skip = c.skip;
  a.skip_background = c.skip_background;
  a.rcv_fw2 = c.cut[0] * c.cut[0];
  a.rcv_mol2 = c.cut[1] * c.cut[1];
  a.rcc2 = c.cut[2] * c.cut[2];
  for (int t = 0; t < 64; ++t) a.grid[t] = (c.grids && t < s->n_types) ? s->grids[t] : nullptr;
  a.ewald_grid = c.grids ? s->grids[s->n_types] : nullptr;
  a.gnx = s->gnx;
  a.gny = s->gny;
  a.gnz = s->gnz;
  for (int i = 0; i < 3; ++i)
    for (int r = 0; r < 3; ++r) a.gic[i][r] = s->gic[i][r];
  a.n_chunks = n_chunks;
  a.chunk = static_cast<int>(chunk);
  a.fw_partners = fw_partners;
  a.partial = s->partial;
  a.counters = s->counters;
  a.out = s->out_mapped;
  a.paired = c.paired ? 1 : 0;
  for (int t = 0; t < 2; ++t)
  {
    a.counts[t] = c.counts[t];
    for (int k = 0; k < 3; ++k) a.cut2[t][k] = c.cut_pair[t][k] * c.cut_pair[t][k];
  }
  a.pockets = s->pockets;
  a.n_pockets = c.pockets_and_field ? s->n_pockets : 0;
  a.pocket_box = s->pocket_box;
  a.ext_on = (c.pockets_and_field && s->ext_on) ? 1 : 0;
  a.ext_type = s->ext_type;
  for (int k = 0; k < 4; ++k) a.ext_geom[k] = s->ext_geom[k];
  a.ext_grid = s->ext_grid;
  a.egnx = s->egnx;
  a.egny = s->egny;
  a.egnz = s->egnz;
  for (int i = 0; i < 3; ++i)
    for (int r = 0; r < 3; ++r) a.egic[i][r] = s->egic[i][r];
  dim3 grid(n_trials, n_chunks);
  kernel<<<grid, kThreads, 0, ctx->stream>>>(a, small);
  RG_CUDA(ctx, cudaGetLastError());
  // the last CTA of each trial wrote its result into mapped pinned memory: completion makes it visible here
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, s->out_host, sizeof(rg_trial_energy) * n_trials);
  return RG_OK;
}

// out = first - second, field by field; the overlap flag is `flag`
void subtractTrials(const rg_trial_energy& x, const rg_trial_energy& y, int32_t flag, rg_trial_energy* out)
{
  rg_trial_energy o{};
  o.framework_vdw = x.framework_vdw - y.framework_vdw;
  o.framework_charge = x.framework_charge - y.framework_charge;
  o.molecule_vdw = x.molecule_vdw - y.molecule_vdw;
  o.molecule_charge = x.molecule_charge - y.molecule_charge;
  for (int g = 0; g < 4; ++g)
  {
    o.dudlambda_vdw[g] = x.dudlambda_vdw[g] - y.dudlambda_vdw[g];
    o.dudlambda_charge[g] = x.dudlambda_charge[g] - y.dudlambda_charge[g];
  }
  o.external_field_vdw = x.external_field_vdw - y.external_field_vdw;
  o.overlap = flag;
  *out = o;
}

// The new atoms and the old atoms of a move as the two sets of a paired call.
rg_status differenceCall(rg_system* s, const rg_atom* new_atoms, int n_new, const rg_atom* old_atoms, int n_old,
                         TrialCall& c, rg_trial_energy* out, std::vector<rg_atom>& packed)
{
  const int stride = std::max(1, std::max(n_new, n_old));
  packed.assign(2 * static_cast<size_t>(stride), rg_atom{});
  if (n_new > 0) std::memcpy(packed.data(), new_atoms, sizeof(rg_atom) * n_new);
  if (n_old > 0) std::memcpy(packed.data() + stride, old_atoms, sizeof(rg_atom) * n_old);
  c.trials = packed.data();
  c.n_trials = 2;
  c.atoms_per_trial = stride;
  c.paired = true;
  c.counts[0] = n_new;
  c.counts[1] = n_old;
  for (int t = 0; t < 2; ++t)
  {
    c.cut_pair[t][0] = s->rc_fw;
    c.cut_pair[t][1] = s->rc_mol;
    c.cut_pair[t][2] = s->rc_coul;
  }
  c.pockets_and_field = false;
  rg_trial_energy res[2];
  rg_status st = runTrials(s, c, res);
  if (st) return st;
  subtractTrials(res[0], res[1], res[0].overlap ? 1 : 0, out);  // only the new atoms can overlap (nullopt)
  return RG_OK;
}
}  // namespace

extern "C"
{
rg_status rg_cbmc_external_energies(rg_system* s, const rg_atom* trials, int n_trials, int atoms_per_trial, int skip,
                                    int64_t skip_background_molecule, double cutoff_framework_vdw,
                                    double cutoff_molecule_vdw, double cutoff_coulomb, rg_trial_energy* out)
{
  if (!s || !trials || !out || n_trials < 0 || atoms_per_trial < 1) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = s->ctx;
  if (atoms_per_trial > kMaxTrialAtoms)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_cbmc_external_energies: at most 64 atoms per trial");
  if (static_cast<long long>(n_trials) * atoms_per_trial > 4096 || n_trials > 4096)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_cbmc_external_energies: at most 4096 trial atoms per call");
  TrialCall c;
  c.trials = trials;
  c.n_trials = n_trials;
  c.atoms_per_trial = atoms_per_trial;
  c.skip = skip;
  c.skip_background = skip_background_molecule;
  c.cut[0] = cutoff_framework_vdw;
  c.cut[1] = cutoff_molecule_vdw;
  c.cut[2] = cutoff_coulomb;
  return runTrials(s, c, out);
}

rg_status rg_cbmc_dual_cutoff_correction(rg_system* s, const rg_atom* trial_set, int n_atoms,
                                         int64_t skip_background_molecule, double dual_cutoff, rg_trial_energy* out)
{
  if (!s || !out || n_atoms < 1 || !trial_set || !(dual_cutoff > 0.0)) return RG_ERR_INVALID_ARGUMENT;
  if (n_atoms > kMaxTrialAtoms)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT, "rg_cbmc_dual_cutoff_correction: at most 64 atoms per set");
  // the set twice: the force field's cutoffs, then the dual cutoff for all three (cbmc/interactions.cpp:214-251)
  std::vector<rg_atom> packed(2 * static_cast<size_t>(n_atoms));
  std::memcpy(packed.data(), trial_set, sizeof(rg_atom) * n_atoms);
  std::memcpy(packed.data() + n_atoms, trial_set, sizeof(rg_atom) * n_atoms);
  TrialCall c;
  c.trials = packed.data();
  c.n_trials = 2;
  c.atoms_per_trial = n_atoms;
  c.skip_background = skip_background_molecule;
  c.paired = true;
  c.counts[0] = c.counts[1] = n_atoms;
  c.cut_pair[0][0] = s->rc_fw;
  c.cut_pair[0][1] = s->rc_mol;
  c.cut_pair[0][2] = s->rc_coul;
  c.cut_pair[1][0] = c.cut_pair[1][1] = c.cut_pair[1][2] = dual_cutoff;
  c.what = "rg_cbmc_dual_cutoff_correction";
  rg_trial_energy res[2];
  rg_status st = runTrials(s, c, res);
  if (st) return st;
  subtractTrials(res[0], res[1], std::max(res[0].overlap, res[1].overlap), out);
  return RG_OK;
}

rg_status rg_framework_molecule_energy_difference(rg_system* s, int charge_method, const rg_atom* new_atoms, int n_new,
                                                  const rg_atom* old_atoms, int n_old, rg_trial_energy* out)
{
  if (!s || !out || n_new < 0 || n_old < 0 || (n_new > 0 && !new_atoms) || (n_old > 0 && !old_atoms))
    return RG_ERR_INVALID_ARGUMENT;
  if (n_new > kMaxTrialAtoms || n_old > kMaxTrialAtoms)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT,
                    "rg_framework_molecule_energy_difference: at most 64 new and 64 old atoms");
  if (charge_method < RG_CHARGE_METHOD_EWALD || charge_method > RG_CHARGE_METHOD_ZERO_DIPOLE)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT, "rg_framework_molecule_energy_difference: bad charge method");
  if (charge_method != RG_CHARGE_METHOD_EWALD && s->ff.use_charge)
    return rg::fail(s->ctx, RG_ERR_UNSUPPORTED,
                    "rg_framework_molecule_energy_difference: charges need the Ewald real-space pair");
  *out = rg_trial_energy{};
  if (n_new == 0 && n_old == 0) return RG_OK;
  TrialCall c;
  c.molecules = false;
  c.grids = charge_method == RG_CHARGE_METHOD_EWALD;  // framework_molecule.cpp:145-146
  c.what = "rg_framework_molecule_energy_difference";
  std::vector<rg_atom> packed;
  return differenceCall(s, new_atoms, n_new, old_atoms, n_old, c, out, packed);
}

rg_status rg_intermolecular_energy_difference(rg_system* s, const rg_atom* new_atoms, int n_new,
                                              const rg_atom* old_atoms, int n_old, rg_trial_energy* out)
{
  if (!s || !out || n_new < 0 || n_old < 0 || (n_new > 0 && !new_atoms) || (n_old > 0 && !old_atoms))
    return RG_ERR_INVALID_ARGUMENT;
  if (n_new > kMaxTrialAtoms || n_old > kMaxTrialAtoms)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT,
                    "rg_intermolecular_energy_difference: at most 64 new and 64 old atoms");
  *out = rg_trial_energy{};
  if (s->omit_inter || (n_new == 0 && n_old == 0)) return RG_OK;  // intermolecular.cpp:207
  TrialCall c;
  c.framework = false;
  c.grids = false;
  c.what = "rg_intermolecular_energy_difference";
  std::vector<rg_atom> packed;
  return differenceCall(s, new_atoms, n_new, old_atoms, n_old, c, out, packed);
}

rg_status rg_system_update_molecules(rg_system* s, int first_atom, const rg_atom* atoms, int n_atoms)
{
  if (!s || first_atom < 0 || n_atoms < 0 || (n_atoms > 0 && !atoms)) return RG_ERR_INVALID_ARGUMENT;
  if (static_cast<long long>(first_atom) + n_atoms > s->n_mol)
    return rg::fail(s->ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_update_molecules: range beyond the stored atoms");
  if (n_atoms == 0) return RG_OK;
  rg_ctx* ctx = s->ctx;
  if (rg_status fs = rg::checkFinite(ctx, atoms, n_atoms, "rg_system_update_molecules")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  RG_CUDA(ctx, cudaMemcpyAsync(s->mol + first_atom, atoms, sizeof(rg_atom) * n_atoms, cudaMemcpyHostToDevice,
                               ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the caller's atom buffer is pageable
  return RG_OK;
}

rg_status rg_system_set_blocked_pockets(rg_system* s, const rg_box* unit_cell, const double* pockets, int n_pockets)
{
  if (!s || n_pockets < 0 || (n_pockets > 0 && (!pockets || !unit_cell))) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = s->ctx;
  for (int i = 0; i < 4 * n_pockets; ++i)
    if (!std::isfinite(pockets[i])) return rg::fail(ctx, RG_ERR_NONFINITE, "rg_system_set_blocked_pockets: NaN or infinite");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (s->pockets) RG_CUDA(ctx, cudaFree(s->pockets));
  s->pockets = nullptr;
  s->n_pockets = 0;
  if (n_pockets == 0) return RG_OK;
  const rg::HostBox hb = rg::makeHostBox(unit_cell);
  std::vector<double4> pk(n_pockets);
  for (int i = 0; i < n_pockets; ++i)
  {
    // the centre in Cartesian: the framework unit cell times the fractions (cbmc/interactions.cpp:33-35)
    const double f[3] = {pockets[4 * i], pockets[4 * i + 1], pockets[4 * i + 2]};
    double r[3];
    rg::matvec(hb.c, f, r);
    pk[i] = make_double4(r[0], r[1], r[2], pockets[4 * i + 3]);
  }
  RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&s->pockets), sizeof(double4) * n_pockets));
  RG_CUDA(ctx, cudaMemcpyAsync(s->pockets, pk.data(), sizeof(double4) * n_pockets, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
    {
      s->pocket_box.c[c][r] = hb.c[c][r];
      s->pocket_box.ic[c][r] = hb.ic[c][r];
    }
  s->pocket_box.triclinic = hb.triclinic ? 1 : 0;
  s->pocket_box.volume = hb.volume;
  s->n_pockets = n_pockets;
  return RG_OK;
}

rg_status rg_system_set_external_field(rg_system* s, int surface_type, const double* geometry, const rg_box* grid_box,
                                       int nx, int ny, int nz, const double* grid, int grid_on_device)
{
  if (!s) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = s->ctx;
  if (surface_type < RG_SURFACE_OFF || surface_type > RG_SURFACE_RECTANGLE_Z)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_set_external_field: bad surface type");
  if (surface_type == RG_SURFACE_GRID_FILE && !grid)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_set_external_field: the grid surface needs a grid");
  if (grid && (!grid_box || nx < 2 || ny < 2 || nz < 2))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_system_set_external_field: grid shape or box");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (s->ext_grid_owned) RG_CUDA(ctx, cudaFree(s->ext_grid));
  s->ext_grid = nullptr;
  s->ext_grid_owned = false;
  s->ext_on = surface_type != RG_SURFACE_OFF;
  s->ext_type = surface_type;
  for (int k = 0; k < 4; ++k) s->ext_geom[k] = geometry ? geometry[k] : 0.0;
  if (grid && s->ext_on)
  {
    const size_t bytes = sizeof(double) * s->scheme * static_cast<size_t>(nx) * ny * nz;
    if (grid_on_device)
      s->ext_grid = const_cast<double*>(grid);
    else
    {
      RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&s->ext_grid), bytes));
      s->ext_grid_owned = true;
      RG_CUDA(ctx, cudaMemcpyAsync(s->ext_grid, grid, bytes, cudaMemcpyHostToDevice, ctx->stream));
      RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    const rg::HostBox hb = rg::makeHostBox(grid_box);
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) s->egic[c][r] = hb.ic[c][r];
    s->egnx = nx;
    s->egny = ny;
    s->egnz = nz;
  }
  return RG_OK;
}
}  // extern "C"

namespace rgd
{
rg_status systemExport(rg_system* s, FF* ff, Box* box, const double** type_grids, const double** ewald_grid,
                       int* n_types, int gdims[3], double gic[3][3], rg_ctx** ctx)
{
  if (!s) return RG_ERR_INVALID_ARGUMENT;
  *ff = s->ff;
  *box = s->box;
  for (int t = 0; t < 64; ++t) type_grids[t] = t < s->n_types ? s->grids[t] : nullptr;
  *ewald_grid = s->grids[s->n_types];
  *n_types = s->n_types;
  gdims[0] = s->gnx;
  gdims[1] = s->gny;
  gdims[2] = s->gnz;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) gic[a][b] = s->gic[a][b];
  *ctx = s->ctx;
  return RG_OK;
}

int systemScheme(const rg_system* s) { return s ? s->scheme : RG_SCHEME_TRICUBIC; }

rg_status systemFramework(rg_system* s, const rg_atom** fw, int* n_fw)
{
  if (!s) return RG_ERR_INVALID_ARGUMENT;
  *fw = s->fw;
  *n_fw = s->n_fw;
  return RG_OK;
}
}  // namespace rgd

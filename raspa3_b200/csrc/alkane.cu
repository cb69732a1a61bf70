// Batched configurational-bias Monte Carlo of flexible chains in many independent systems (rg_alkane_*).
//
// Every system of the batch is advanced by one thread-block cluster of a persistent kernel. The cluster's CTAs hold
// the system's framework atoms, split between them, and a full copy of its molecules in shared memory for all moves
// of a launch; positions are fixed-point fractional coordinates (uint32 per axis), so the difference of two positions
// wraps to the minimum image exactly and converts to an FP32 Cartesian displacement with a relative error of 2^-24,
// independent of the box size. Each CTA evaluates the pair terms of its slice of partners in FP32 (one per-thread
// FP32 partial per bead), the partials are reduced in FP64 across warps, and the CTAs exchange per-bead sums through
// distributed shared memory. Every CTA of a cluster draws the same counter-based random numbers and takes the same
// decisions, so no decision is ever broadcast: only the partial energies cross the cluster.
//
// Reference algorithm per system (file:line in the RASPA3 source tree):
//   moves             mc_moves/component/translation.cpp:30-200, insertion_cbmc.cpp:34-207, deletion_cbmc.cpp:34-195
//   first bead        cbmc/multiple_first_bead.cpp:20-76
//   chain             cbmc/flexible_molecules/insertion.cpp:32-126, deletion.cpp:30-104
//   trials            cbmc/operators.cpp:951-1078 (seed step, base conformation, selectTorsionOrientation :135-196)
//   trial energies    cbmc/interactions.cpp:54-179 -> interactions_framework_molecule.cpp, interactions_intermolecular.cpp
// The base conformation of a step is drawn exactly from the distribution that the reference's internal bond/bend
// Metropolis Monte Carlo (operators.cpp:203-447) converges to, p(theta) ~ sin(theta) exp(-beta U_bend(theta)) with a
// uniform azimuth (the reference's own comment at system.ixx:593-600 notes that this MC targets exp(-beta U_intra)
// whatever its seed): a Gaussian proposal around theta0 accepted with probability sin(theta), 32 proposals per warp
// round. This replaces a serial chain of 2*2*150 dependent updates per step by one warp vote.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "rng.cuh"

namespace cg = cooperative_groups;

namespace
{
constexpr int kMaxBeads = 8;
constexpr int kMaxTrials = 16;
constexpr int kMaxTorsion = 128;
constexpr int kMaxMolecules = 256;
constexpr int kMaxTypes = 16;
constexpr int kMaxWarps = 16;  // up to 512 threads per CTA
constexpr int kStats = 24;    // the rg_gcmc_chain_result record of gcmc.cu
constexpr double kMinimumRosenbluth = 1e-150;  // ForceField::minimumRosenbluthFactor (forcefield.ixx:143)
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr float kFix = 2.3283064365386963e-10f;  // 2^-32

struct SysDev
{
  double c[3][3];   // cell, c[col][row]
  double ic[3][3];  // inverse
  float hf[3][3];   // cell in FP32 for displacements
  int triclinic;
  double volume, beta, fugacity, w_ig, max_translation, p_translation, p_swap;
  int fw_offset, n_fw, max_molecules, pos_offset;
  int nb, n_first, n_dir, n_tors;
  int types[kMaxBeads];
  double bond, bend_k, bend_theta0, sigma_theta, torsion[4];
};

struct Ctrl
{
  int record;
  int pad;
  long long block_len;
};

struct Params
{
  const SysDev* sys;
  const int4* fw;        // fixed-point framework atoms, .w = type
  double* pos;           // 3 doubles per bead, system s at sys[s].pos_offset
  int* n_mol;
  double* energy;
  long long* move_base;
  double* stats;         // [s][kStats]
  unsigned long long* pairs;  // [s]: in-cutoff pair evaluations (the algorithmic unit of the trial energies)
  const Ctrl* ctrl;
  const float4* ljf;     // [kMaxTypes][kMaxTypes]: 4 eps, sigma^2, shift, 0 (FP32 pair terms)
  const double2* ljd;    // [kMaxTypes][kMaxTypes]: 4 eps, sigma^2 (FP64 intra-molecular terms)
  float rc2_fw, rc2_mm, overlap_f;
  unsigned long long seed;
};

// random slots: [31:28] kind, [27:24] step, [23:16] index, [15:0] sub
__host__ __device__ constexpr uint32_t slot(uint32_t kind, uint32_t step, uint32_t index, uint32_t sub)
{
  return (kind << 28) | (step << 24) | (index << 16) | sub;
}
enum : uint32_t
{
  kKindMove = 1,
  kKindFirst = 2,
  kKindDir = 3,
  kKindTheta = 4,
  kKindSpin = 5,
  kKindSelect = 6
};

// the cluster a CTA belongs to: cluster calls are made only when C > 1 (single-CTA kernels never touch them)
struct Cl
{
  int rank, C;
};

struct Shared
{
  float4 tab[kMaxTypes * kMaxTypes];
  int4 bead[kMaxTrials];  // beads evaluated (fixed point, .w = type)
  double red[2][32 * kMaxWarps];  // per-thread framework / molecule partial sums
  unsigned red_ovl[kMaxWarps];
  double xch[2][2 * kMaxTrials];  // per-CTA sums exchanged across the cluster (double-buffered)
  unsigned xch_ovl[2];
  double efw[kMaxTrials], emm[kMaxTrials];
  unsigned ovl;
  double3 x[kMaxBeads];    // chain being grown / retraced (Cartesian)
  double3 old[kMaxBeads];  // molecule being retraced or translated
  double3 dir[kMaxTrials];
  double tw[kMaxTrials];
  double intra[kMaxTrials];
  double theta[kMaxBeads], psi[kMaxBeads];   // base-conformation bend angle and azimuth / pi per step (insertion)
  double tD[kMaxBeads];                      // retrace: cosine of the old dihedral at step j
  double ttw[kMaxBeads][kMaxTrials];         // torsion weight per step and direction
  int tsel[kMaxBeads][kMaxTrials];           // selected spin per step and direction
  double W, eext, dU, stats[kStats];
  int fail, kind, m, axis, n, accept;
  unsigned long long pairs;
  double energy, disp, u_acc;
};

__device__ __forceinline__ double2 urand(const Params& p, int s, long long move, uint32_t sl)
{
  return rgd::uniform2(p.seed, s, move, sl);
}

__device__ __forceinline__ double3 d3(double x, double y, double z) { return make_double3(x, y, z); }
__device__ __forceinline__ double3 add(double3 a, double3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ double3 sub(double3 a, double3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 scale(double s, double3 a) { return d3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 cross(double3 a, double3 b)
{
  return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double3 normalized(double3 a) { return scale(1.0 / sqrt(dot(a, a)), a); }

// double3::rotateAroundAxis (mathkit/double3.ixx:163-178): rotates v about the unit axis a by the angle whose sine
// and cosine are s and c
__device__ __forceinline__ double3 rotateAroundSC(double3 a, double3 v, double s, double c)
{
  const double w = 1.0 - c;
  return d3(v.x * (a.x * a.x * w + c) + v.y * (a.x * a.y * w + a.z * s) + v.z * (a.x * a.z * w - a.y * s),
            v.x * (a.x * a.y * w - a.z * s) + v.y * (a.y * a.y * w + c) + v.z * (a.y * a.z * w + a.x * s),
            v.x * (a.x * a.z * w + a.y * s) + v.y * (a.y * a.z * w - a.x * s) + v.z * (a.z * a.z * w + c));
}

// fixed-point fractional position (each coordinate in [0,1) scaled by 2^32)
__device__ __forceinline__ uint32_t fixOf(double s)
{
  s -= floor(s);
  return static_cast<uint32_t>(static_cast<unsigned long long>(s * 4294967296.0));
}
__device__ __forceinline__ int4 toFixed(const SysDev& S, double3 r, int w)
{
  const double s0 = S.ic[0][0] * r.x + S.ic[1][0] * r.y + S.ic[2][0] * r.z;
  const double s1 = S.ic[0][1] * r.x + S.ic[1][1] * r.y + S.ic[2][1] * r.z;
  const double s2 = S.ic[0][2] * r.x + S.ic[1][2] * r.y + S.ic[2][2] * r.z;
  return make_int4(static_cast<int>(fixOf(s0)), static_cast<int>(fixOf(s1)), static_cast<int>(fixOf(s2)), w);
}

// BendPotential::calculateEnergy, harmonic (bend_potential.cpp:321-380)
__device__ __forceinline__ double bendEnergy(const SysDev& S, double3 a, double3 b, double3 c)
{
  const double3 ab = normalized(sub(a, b)), cb = normalized(sub(c, b));
  const double ct = fmin(1.0, fmax(-1.0, dot(ab, cb)));
  const double th = acos(ct) - S.bend_theta0;
  return 0.5 * S.bend_k * th * th;
}

// TorsionPotential::calculateEnergy, TraPPE (torsion_potential.cpp:393-476)
__device__ __forceinline__ double torsionEnergy(const SysDev& S, double3 a, double3 b, double3 c, double3 d)
{
  const double3 dab = sub(a, b), dcb = normalized(sub(c, b)), ddc = sub(d, c);
  const double3 dr = normalized(sub(dab, scale(dot(dab, dcb), dcb)));
  const double3 ds = normalized(sub(ddc, scale(dot(ddc, dcb), dcb)));
  const double cp = fmin(1.0, fmax(-1.0, dot(dr, ds)));
  const double* p = S.torsion;
  return p[0] + (1.0 + cp) * (p[1] + p[3] - 2.0 * (cp - 1.0) * (p[2] - 2.0 * p[3] * cp));
}

// intra-molecular Lennard-Jones of bead j at r with beads k <= j - 4 (van_der_waals_potential.cpp:43-62, no cut-off)
__device__ __forceinline__ double intraVdw(const Params& p, const SysDev& S, const double3* x, int j, double3 r)
{
  double e = 0.0;
  for (int k = 0; k + 4 <= j; ++k)
  {
    const double3 d = sub(r, x[k]);
    const double2 q = p.ljd[S.types[k] * kMaxTypes + S.types[j]];
    const double rri = q.y / dot(d, d);
    const double t = rri * rri * rri;
    e += q.x * (t * (t - 1.0));
  }
  return e;
}

// all internal terms of a chain: bends, torsions, intra-molecular VDW (bonds are fixed)
__device__ __noinline__ double internalEnergy(const Params& p, const SysDev& S, const double3* x)
{
  double e = 0.0;
  for (int j = 2; j < S.nb; ++j) e += bendEnergy(S, x[j - 2], x[j - 1], x[j]);
  for (int j = 3; j < S.nb; ++j) e += torsionEnergy(S, x[j - 3], x[j - 2], x[j - 1], x[j]);
  for (int j = 4; j < S.nb; ++j) e += intraVdw(p, S, x, j, x[j]);
  return e;
}

// Trial selection by one warp, lane i holding trial i (i < 32): *sum = sum over the non-overlapping trials of
// exp(lbf) (the Rosenbluth sum), and the index chosen by CBMC::selectTrialPosition (cbmc/util.cpp:14-47): the first
// trial whose cumulative shifted Boltzmann factor reaches u times the total. retrace: trial 0 (the old position).
// Returns -1 when every trial overlaps. Called by all 32 lanes of warp 0.
__device__ __forceinline__ int warpSelect(double lbf, bool ok, bool retrace, double u, double* sum)
{
  const int lane = threadIdx.x & 31;
  const unsigned okMask = __ballot_sync(0xffffffffu, ok);
  double mx = ok ? lbf : -1e300;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  double direct = ok ? exp(lbf) : 0.0;
  const double shifted = ok ? exp(lbf - mx) : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) direct += __shfl_xor_sync(0xffffffffu, direct, o);
  double incl = shifted;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    const double t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const double total = __shfl_sync(0xffffffffu, incl, 31);
  *sum = direct;
  if (okMask == 0u) return -1;
  if (retrace) return 0;
  const unsigned hit = __ballot_sync(0xffffffffu, ok && incl >= u * total);
  return hit ? __ffs(hit) - 1 : 31 - __clz(okMask);
}

// Squared distance of bead B and partner P in FP32 from their exact fixed-point displacement (the uint32 wrap is the
// minimum image).
template <bool TRI>
__device__ __forceinline__ float beadDistance2(const SysDev& S, int4 B, int4 P)
{
  const float f0 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.x) - static_cast<uint32_t>(P.x))) * kFix;
  const float f1 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.y) - static_cast<uint32_t>(P.y))) * kFix;
  const float f2 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.z) - static_cast<uint32_t>(P.z))) * kFix;
  float rx, ry, rz;
  if (TRI)
  {
    rx = fmaf(S.hf[0][0], f0, fmaf(S.hf[1][0], f1, S.hf[2][0] * f2));
    ry = fmaf(S.hf[0][1], f0, fmaf(S.hf[1][1], f1, S.hf[2][1] * f2));
    rz = fmaf(S.hf[0][2], f0, fmaf(S.hf[1][2], f1, S.hf[2][2] * f2));
  }
  else
  {
    rx = S.hf[0][0] * f0;
    ry = S.hf[1][1] * f1;
    rz = S.hf[2][2] * f2;
  }
  return fmaf(rx, rx, fmaf(ry, ry, rz * rz));
}

__device__ __forceinline__ void beadPairEnergy(const Shared& sh, int bt, int4 P, float r2, float rc2, float ovlf,
                                               double& acc, unsigned& ovl, unsigned& inside, int b)
{
  if (r2 < rc2)
  {
    const float4 q = sh.tab[bt + (P.w & 0xff)];
    const float t = q.y * __frcp_rn(r2);
    const float t3 = t * t * t;
    const float e = q.x * (t3 * (t3 - 1.0f)) - q.z;
    acc += static_cast<double>(e);
    inside += 1u;
    if (e > ovlf) ovl |= 1u << b;
  }
}

// Lennard-Jones energy of bead B with partners[begin], partners[begin + stride], .. (fixed point), FP32 from the exact
// displacement, accumulated in FP64 in partner order. Four partners per iteration: their distances without branches
// (a skipped molecule's at infinity), then the energies of those within the cutoff. Bit b of ovl is set if a pair
// exceeds the overlap criterion.
template <bool TRI, bool SKIP>
__device__ __forceinline__ void beadPartners(const Shared& sh, const SysDev& S, int4 B, const int4* partners,
                                             int begin, int n, int stride, int skip, float rc2, float ovlf,
                                             double& acc, unsigned& ovl, unsigned& inside, int b)
{
  const int bt = (B.w & 0xff) * kMaxTypes;
  int i = begin;
  for (; i + 3 * stride < n; i += 4 * stride)
  {
    const int4 P0 = partners[i], P1 = partners[i + stride], P2 = partners[i + 2 * stride], P3 = partners[i + 3 * stride];
    const float r0 = SKIP && (P0.w >> 8) == skip ? INFINITY : beadDistance2<TRI>(S, B, P0);
    const float r1 = SKIP && (P1.w >> 8) == skip ? INFINITY : beadDistance2<TRI>(S, B, P1);
    const float r2 = SKIP && (P2.w >> 8) == skip ? INFINITY : beadDistance2<TRI>(S, B, P2);
    const float r3 = SKIP && (P3.w >> 8) == skip ? INFINITY : beadDistance2<TRI>(S, B, P3);
    if (fminf(fminf(r0, r1), fminf(r2, r3)) < rc2)
    {
      beadPairEnergy(sh, bt, P0, r0, rc2, ovlf, acc, ovl, inside, b);
      beadPairEnergy(sh, bt, P1, r1, rc2, ovlf, acc, ovl, inside, b);
      beadPairEnergy(sh, bt, P2, r2, rc2, ovlf, acc, ovl, inside, b);
      beadPairEnergy(sh, bt, P3, r3, rc2, ovlf, acc, ovl, inside, b);
    }
  }
  for (; i < n; i += stride)
  {
    const int4 P = partners[i];
    if (SKIP && (P.w >> 8) == skip) continue;
    beadPairEnergy(sh, bt, P, beadDistance2<TRI>(S, B, P), rc2, ovlf, acc, ovl, inside, b);
  }
}

// Framework + molecule energies of the nbd beads in sh.bead, summed over the cluster into sh.efw / sh.emm / sh.ovl.
// Thread t works on bead t % nbd with partner stream t / nbd: the framework slice of this CTA is fwS[0, nfw), the
// molecule beads molS[0, nmb) are interleaved over the cluster ranks. The per-thread sums are reduced per bead in a
// fixed order (within a warp lanes l, l + nbd, .. by shuffles, then the warps in order), the CTAs' sums in rank
// order, so every CTA ends with identical totals. Called by every thread of every CTA of the cluster.
__device__ __noinline__ void evalBeads(Shared& sh, const Params& p, const SysDev& S, const int4* fwS, int nfw, const int4* molS,
                          int nmb, int nbd, int skip, Cl cl, int& eval)
{
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = T >> 5;
  const int rank = cl.rank, C = cl.C;
  const int streams = T / nbd, b = tid % nbd, st = tid / nbd;
  double afw = 0.0, amm = 0.0;
  unsigned ovl = 0, inside = 0;
  if (st < streams)
  {
    const int4 B = sh.bead[b];
    if (S.triclinic)
    {
      beadPartners<true, false>(sh, S, B, fwS, st, nfw, streams, -1, p.rc2_fw, p.overlap_f, afw, ovl, inside, b);
      beadPartners<true, true>(sh, S, B, molS, rank * streams + st, nmb, C * streams, skip, p.rc2_mm, p.overlap_f,
                               amm, ovl, inside, b);
    }
    else
    {
      beadPartners<false, false>(sh, S, B, fwS, st, nfw, streams, -1, p.rc2_fw, p.overlap_f, afw, ovl, inside, b);
      beadPartners<false, true>(sh, S, B, molS, rank * streams + st, nmb, C * streams, skip, p.rc2_mm, p.overlap_f,
                                amm, ovl, inside, b);
    }
  }
  // lane l < nbd ends with its warp's sums of bead (32 warp + l) mod nbd (threads past the last stream add zeros)
  const double ownf = afw, ownm = amm;
  for (int o = nbd; nbd > 0 && o < 32; o += nbd)
  {
    const double yf = __shfl_down_sync(0xffffffffu, ownf, o), ym = __shfl_down_sync(0xffffffffu, ownm, o);
    if (lane + o < 32)
    {
      afw += yf;
      amm += ym;
    }
  }
  if (lane < nbd)
  {
    const int bb = (32 * warp + lane) % nbd;
    sh.red[0][warp * kMaxTrials + bb] = afw;
    sh.red[1][warp * kMaxTrials + bb] = amm;
  }
  inside = __reduce_add_sync(0xffffffffu, inside);
  if (lane == 0 && inside) atomicAdd(&sh.pairs, static_cast<unsigned long long>(inside));
  ovl = __reduce_or_sync(0xffffffffu, ovl);
  if (lane == 0) sh.red_ovl[warp] = ovl;
  __syncthreads();
  const int buf = eval & 1;
  eval += 1;
  // thread t < 16 sums the framework part of bead t, thread 16 + t its molecule part, over the warps in order; a
  // lone CTA writes its totals at once
  double sum = 0.0;
  const int which = tid >= kMaxTrials, bb = tid - which * kMaxTrials;
  if (tid < 2 * kMaxTrials && bb < nbd)
    for (int w = 0; w < nw; ++w) sum += sh.red[which][w * kMaxTrials + bb];
  unsigned octa = 0;
  if (tid == 2 * kMaxTrials)
    for (int w = 0; w < nw; ++w) octa |= sh.red_ovl[w];
  if (C == 1)
  {
    if (tid < kMaxTrials) sh.efw[tid] = sum;
    if (tid >= kMaxTrials && tid < 2 * kMaxTrials) sh.emm[tid - kMaxTrials] = sum;
    if (tid == 2 * kMaxTrials) sh.ovl = octa;
  }
  else
  {
    if (tid < 2 * kMaxTrials) sh.xch[buf][tid] = sum;
    if (tid == 2 * kMaxTrials) sh.xch_ovl[buf] = octa;
    // every CTA's sums are complete before any is read; sums are taken in rank order, identical in every CTA
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (tid < 2 * kMaxTrials)
    {
      double sum = 0.0;
      for (int q = 0; q < C; ++q) sum += cluster.map_shared_rank(&sh.xch[buf][0], q)[tid];
      if (tid < kMaxTrials)
        sh.efw[tid] = sum;
      else
        sh.emm[tid - kMaxTrials] = sum;
    }
    if (tid == 2 * kMaxTrials)
    {
      unsigned o = 0;
      for (int q = 0; q < C; ++q) o |= cluster.map_shared_rank(&sh.xch_ovl[0], q)[buf];
      sh.ovl = o;
    }
  }
  __syncthreads();
}

// Four spin angles per Philox draw: word k of draw (j, i, q) gives spin 4q + k of direction i at step j, the angle
// (2u - 1) pi with u = (word + 1/2) 2^-32; sincospi returns its sine and cosine.
__device__ __forceinline__ uint4 spinWords(const Params& p, int s, long long move, int j, int i, int q)
{
  uint32_t c[4] = {slot(kKindSpin, j, i, q), static_cast<uint32_t>(move), static_cast<uint32_t>(move >> 32),
                   static_cast<uint32_t>(s)};
  rgd::philox(c, static_cast<uint32_t>(p.seed), static_cast<uint32_t>(p.seed >> 32));
  return make_uint4(c[0], c[1], c[2], c[3]);
}
__device__ __forceinline__ void spinAngle(uint32_t word, double* sa, double* ca)
{
  const double u = (static_cast<double>(word) + 0.5) * 0x1.0p-32;
  sincospi(2.0 * u - 1.0, sa, ca);
}

// TraPPE torsion energy from the torsion cosine (torsion_potential.cpp:464-473)
__device__ __forceinline__ double trappe(const SysDev& S, double cp)
{
  const double* q = S.torsion;
  return q[0] + (1.0 + cp) * (q[1] + q[3] - 2.0 * (cp - 1.0) * (q[2] - 2.0 * q[3] * cp));
}

// Signed dihedral (cos D, sin D) about the unit axis a = normalized(x2 - x3) of the position y grown from x3, with
// reference atom x1 (the torsion x1-x2-x3-y): cos D is TorsionPotential's cos(phi), and a spin of y by alpha about a
// (rotateAroundAxis) turns D into D - alpha.
__device__ __forceinline__ void signedDihedral(double3 x1, double3 x2, double3 x3, double3 y, double3 a, double* cD,
                                               double* sD)
{
  const double3 dcb = scale(-1.0, a);
  const double3 dab = sub(x1, x2), ddc = sub(y, x3);
  const double3 dr = normalized(sub(dab, scale(dot(dab, dcb), dcb)));
  const double3 ds = normalized(sub(ddc, scale(dot(ddc, dcb), dcb)));
  *cD = dot(dr, ds);
  *sD = dot(cross(dr, ds), a);
}

// Everything of a growth or retrace that does not depend on where the chain goes, done once per move by the warps
// in parallel (no barrier inside):
//  * insertion: the bend angle and azimuth of every step j >= 2, drawn exactly from sin(theta) exp(-beta U_bend) by
//    a warp vote over Gaussian proposals;
//  * every step j >= 3 and direction i: the coupled-decoupled torsion selection of selectTorsionOrientation
//    (operators.cpp:135-196). A spin by a uniform angle alpha about the bond gives the dihedral D - alpha, itself
//    uniform whatever D is, so the spins are drawn directly as uniform dihedrals phi: the torsion weight
//    (1/n) sum exp(-beta U(phi_s)) and the selected phi do not depend on the chain; the step then turns its base by
//    alpha = D - phi_sel. In a retrace, spin 0 of direction 0 is the old dihedral itself (sh.tD holds its cosine).
//  * step 2 has no torsion: its weight is 1 and its spin is uniform.
__device__ __noinline__ void precomputeGrowth(Shared& sh, const Params& p, const SysDev& S, int s, long long move, bool retrace)
{
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  const int nb = S.nb, kd = S.n_dir, nt = S.n_tors;
  const double beta = S.beta;
  const int nTheta = retrace ? 0 : max(0, nb - 2);
  const int nTors = max(0, nb - 2) * kd;  // steps j = 2..nb-1
  for (int task = warp; task < nTheta + nTors; task += nw)
  {
    if (task < nTheta)
    {
      const int j = 2 + task;
      double theta = S.bend_theta0, psi = 0.0;
      for (int round = 0; round < 64; ++round)
      {
        const double2 u = urand(p, s, move, slot(kKindTheta, j, round, 2 * lane));
        const double2 v = urand(p, s, move, slot(kKindTheta, j, round, 2 * lane + 1));
        const double g = sqrt(-2.0 * log(1.0 - u.x)) * cospi(2.0 * u.y);
        const double th = S.bend_theta0 + S.sigma_theta * g;
        const bool ok = th > 0.0 && th < kPi && v.x < sinpi(th / kPi);
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (bal)
        {
          const int l = __ffs(bal) - 1;
          theta = __shfl_sync(0xffffffffu, th, l);
          psi = 2.0 * __shfl_sync(0xffffffffu, v.y, l);  // azimuth / pi
          break;
        }
      }
      if (lane == 0)
      {
        sh.theta[j] = theta;
        sh.psi[j] = psi;
      }
      continue;
    }
    const int t = task - nTheta, j = 2 + t / kd, i = t - (j - 2) * kd;
    if (j == 2)
    {
      // no torsion: all spins weigh 1; the selected one is uniform
      if (lane == 0)
      {
        sh.ttw[j][i] = 1.0;
        sh.tsel[j][i] = static_cast<int>(urand(p, s, move, slot(kKindSelect, j, i, 0)).x * nt) % nt;
      }
      continue;
    }
    // lane owns spins 4 lane .. 4 lane + 3 (one Philox draw, four 32-bit words)
    double lbf[4];
    const uint4 w = spinWords(p, s, move, j, i, lane);
    const uint32_t words[4] = {w.x, w.y, w.z, w.w};
    double mx = -1e300;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
      const int sp = 4 * lane + k;
      lbf[k] = -1e300;
      if (sp < nt)
      {
        const double cp = (retrace && i == 0 && sp == 0)
                              ? sh.tD[j]
                              : cospi(2.0 * ((static_cast<double>(words[k]) + 0.5) * 0x1.0p-32) - 1.0);
        lbf[k] = -beta * trappe(S, fmin(1.0, fmax(-1.0, cp)));
        mx = fmax(mx, lbf[k]);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    double e[4], local = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
      e[k] = (4 * lane + k < nt) ? exp(lbf[k] - mx) : 0.0;
      local += e[k];
    }
    double incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
      const double v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const double total = __shfl_sync(0xffffffffu, incl, 31);
    int sel = 0;
    if (!(retrace && i == 0))
    {
      const double target = urand(p, s, move, slot(kKindSelect, j, i, 0)).x * total;
      const unsigned bal = __ballot_sync(0xffffffffu, incl >= target && local > 0.0);
      const int l = bal ? __ffs(bal) - 1 : 31;
      int mine = -1;
      if (lane == l)
      {
        double cum = incl - local;
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
          if (4 * lane + k >= nt || mine >= 0) continue;
          cum += e[k];
          if (cum >= target) mine = 4 * lane + k;
        }
        if (mine < 0) mine = min(4 * lane + 3, nt - 1);
      }
      sel = __shfl_sync(0xffffffffu, mine, l);
    }
    if (lane == 0)
    {
      sh.ttw[j][i] = exp(mx) * total / static_cast<double>(nt);
      sh.tsel[j][i] = sel;
    }
  }
}

// Trial positions of step j >= 2 from the precomputed selections: direction i turns the step's base by
// alpha = D - phi_sel (retrace: direction 0 is the old position). Threads i < kd; ends with a barrier.
__device__ __noinline__ void stepTrials(Shared& sh, const Params& p, const SysDev& S, int s, long long move, int j, bool retrace)
{
  const int tid = threadIdx.x;
  if (tid < S.n_dir)
  {
    const int i = tid;
    const double3 cur = sh.x[j - 1];
    const double3 a = normalized(sub(sh.x[j - 2], cur));
    double3 base;
    if (retrace)
      base = sh.old[j];
    else
    {
      // direction at angle theta from a with azimuth psi about a
      const double3 h = fabs(a.x) < 0.6 ? d3(1, 0, 0) : (fabs(a.y) < 0.6 ? d3(0, 1, 0) : d3(0, 0, 1));
      const double3 e1 = normalized(cross(a, h));
      const double3 e2 = cross(a, e1);
      double sp, cp, st, ct;
      sincospi(sh.psi[j], &sp, &cp);
      sincospi(sh.theta[j] / kPi, &st, &ct);
      base = add(cur, scale(S.bond, add(scale(ct, a), scale(st, add(scale(cp, e1), scale(sp, e2))))));
    }
    double3 pos;
    if (retrace && i == 0)
      pos = sh.old[j];
    else
    {
      const int sel = sh.tsel[j][i];
      const uint4 w = spinWords(p, s, move, j, i, sel >> 2);
      const uint32_t words[4] = {w.x, w.y, w.z, w.w};
      double sphi, cphi;
      spinAngle(words[sel & 3], &sphi, &cphi);
      double sa = sphi, ca = cphi;  // step 2: any uniform angle (no dihedral)
      if (j >= 3)
      {
        double cD, sD;
        signedDihedral(sh.x[j - 3], sh.x[j - 2], cur, base, a, &cD, &sD);
        ca = cD * cphi + sD * sphi;  // cos(D - phi)
        sa = sD * cphi - cD * sphi;  // sin(D - phi)
      }
      pos = add(cur, rotateAroundSC(a, sub(base, cur), sa, ca));
    }
    sh.dir[i] = pos;
    sh.tw[i] = sh.ttw[j][i];
    sh.bead[i] = toFixed(S, pos, S.types[j]);
  }
  __syncthreads();
}

// One growth (insertion: retrace = false) or retrace of molecule m (its positions in sh.old). On return sh.fail,
// sh.W (Rosenbluth weight), sh.eext (external energy of the chain) and sh.x (grown chain) are set.
__device__ __noinline__ void growChain(Shared& sh, const Params& p, const SysDev& S, int s, long long move, bool retrace, int m,
                          const int4* fwS, int nfw, const int4* molS, int nmb, Cl cl, int& eval)
{
  const int tid = threadIdx.x;
  const double beta = S.beta;
  const int skip = retrace ? m : -1;
  const int k1 = S.n_first, kd = S.n_dir, nb = S.nb;
  if (retrace && tid >= 3 && tid < nb)
  {
    // the old dihedral of every step (spin 0 of direction 0 of the retrace)
    const int j = tid;
    double cD, sD;
    signedDihedral(sh.old[j - 3], sh.old[j - 2], sh.old[j - 1], sh.old[j],
                   normalized(sub(sh.old[j - 2], sh.old[j - 1])), &cD, &sD);
    sh.tD[j] = cD;
  }
  __syncthreads();
  precomputeGrowth(sh, p, S, s, move, retrace);
  // first bead (multiple_first_bead.cpp:20-76)
  if (tid < k1)
  {
    double3 r;
    int4 f;
    if (retrace && tid == 0)
    {
      r = sh.old[0];
      f = toFixed(S, r, S.types[0]);
    }
    else
    {
      const double2 u = urand(p, s, move, slot(kKindFirst, 0, tid, 0));
      const double u2 = urand(p, s, move, slot(kKindFirst, 0, tid, 1)).x;
      r = d3(S.c[0][0] * u.x + S.c[1][0] * u.y + S.c[2][0] * u2, S.c[0][1] * u.x + S.c[1][1] * u.y + S.c[2][1] * u2,
             S.c[0][2] * u.x + S.c[1][2] * u.y + S.c[2][2] * u2);
      f = make_int4(static_cast<int>(fixOf(u.x)), static_cast<int>(fixOf(u.y)), static_cast<int>(fixOf(u2)),
                    S.types[0]);
    }
    sh.dir[tid] = r;
    sh.bead[tid] = f;
  }
  __syncthreads();
  evalBeads(sh, p, S, fwS, nfw, molS, nmb, k1, skip, cl, eval);
  if (tid < 32)
  {
    const bool ok = tid < k1 && !((sh.ovl >> tid) & 1u);
    const double lbf = ok ? -beta * (sh.efw[tid] + sh.emm[tid]) : 0.0;
    double sum;
    const int sel = warpSelect(lbf, ok, retrace, urand(p, s, move, slot(kKindMove, 0, 0, 3)).x, &sum);
    if (tid == 0)
    {
      sh.fail = (sel < 0) || (retrace && ((sh.ovl & 1u) != 0u));
      if (!sh.fail)
      {
        sh.W = sum / static_cast<double>(k1);
        sh.x[0] = sh.dir[sel];
        sh.eext = sh.efw[sel] + sh.emm[sel];
      }
    }
  }
  __syncthreads();
  if (sh.fail) return;
  double Wc = 1.0;  // chain weight (thread 0)
  for (int j = 1; j < nb; ++j)
  {
    if (j == 1)
    {
      // seed step (operators.cpp:994-1004): fixed bond length, uniform direction
      if (tid < kd)
      {
        double3 r;
        if (retrace && tid == 0)
          r = sh.old[1];
        else
        {
          const double2 u = urand(p, s, move, slot(kKindDir, 1, tid, 0));
          const double z = 1.0 - 2.0 * u.x, rr = sqrt(fmax(0.0, 1.0 - z * z));
          double sp, cp;
          sincospi(2.0 * u.y, &sp, &cp);
          r = add(sh.x[0], scale(S.bond, d3(rr * cp, rr * sp, z)));
        }
        sh.dir[tid] = r;
        sh.tw[tid] = 1.0;
        sh.bead[tid] = toFixed(S, r, S.types[1]);
      }
      __syncthreads();
    }
    else
    {
      stepTrials(sh, p, S, s, move, j, retrace);
    }
    evalBeads(sh, p, S, fwS, nfw, molS, nmb, kd, skip, cl, eval);
    if (tid < 32)
    {
      const bool ok = tid < kd && !((sh.ovl >> tid) & 1u);
      const double intra = (ok && j >= 4) ? intraVdw(p, S, sh.x, j, sh.dir[tid]) : 0.0;
      const double lbf = ok ? -beta * (sh.efw[tid] + sh.emm[tid] + intra) : 0.0;
      double sum;
      const int sel = warpSelect(lbf, ok, retrace, urand(p, s, move, slot(kKindSelect, j, 255, 0)).x, &sum);
      if (tid == 0)
      {
        sh.fail = (sel < 0) || (retrace && ((sh.ovl & 1u) != 0u));
        if (!sh.fail)
        {
          Wc *= sh.tw[sel] * sum / static_cast<double>(kd);
          if (!retrace && Wc < kMinimumRosenbluth) sh.fail = 1;
          sh.x[j] = sh.dir[sel];
          sh.eext += sh.efw[sel] + sh.emm[sel];
        }
        if (j == nb - 1 && !sh.fail) sh.W *= Wc;
      }
    }
    __syncthreads();
    if (sh.fail) return;
  }
}

__device__ __forceinline__ int4* dynamicBase(unsigned char* smem)
{
  return reinterpret_cast<int4*>(smem + ((sizeof(Shared) + 15) & ~static_cast<size_t>(15)));
}

// The persistent Monte Carlo kernel: one cluster per system, `moves` move attempts per system.
template <int T>
__global__ void __launch_bounds__(T, 1) alkaneKernel(Params p, const int* __restrict__ order, int fw_cap, int moves)
{
  extern __shared__ __align__(16) unsigned char smem[];
  Shared& sh = *reinterpret_cast<Shared*>(smem);
  int4* fwS = dynamicBase(smem);
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = static_cast<int>(cluster.block_rank()), C = static_cast<int>(cluster.num_blocks());
  const Cl cl{rank, C};
  const int s = order[blockIdx.x / C];
  const SysDev& S = p.sys[s];
  int4* molS = fwS + fw_cap;
  const int tid = threadIdx.x;
  const int nb = S.nb;

  const int per = (S.n_fw + C - 1) / C, f0 = rank * per;
  const int nfw = max(0, min(S.n_fw, f0 + per) - f0);
  for (int i = tid; i < nfw; i += T) fwS[i] = p.fw[S.fw_offset + f0 + i];
  for (int i = tid; i < kMaxTypes * kMaxTypes; i += T) sh.tab[i] = p.ljf[i];
  double* pos = p.pos + 3ll * S.pos_offset;
  const int n0 = p.n_mol[s];
  for (int i = tid; i < n0 * nb; i += T)
  {
    const int m = i / nb, b = i - m * nb;
    molS[i] = toFixed(S, d3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), S.types[b] | (m << 8));
  }
  const int record = p.ctrl->record;
  const long long block_len = p.ctrl->block_len;
  double* st = p.stats + static_cast<long long>(s) * kStats;
  if (tid == 0)
  {
    sh.n = n0;
    sh.energy = p.energy[s];
    sh.pairs = 0ull;
    for (int k = 0; k < kStats; ++k) sh.stats[k] = st[k];
  }
  const long long move0 = p.move_base[s];
  int eval = 0;  // evaluation counter (selects the exchange buffer), identical in every thread
  __syncthreads();

  for (int mv = 0; mv < moves; ++mv)
  {
    const long long move = move0 + mv;
    if (tid == 0)
    {
      const double2 u0 = urand(p, s, move, slot(kKindMove, 0, 0, 0));
      const double2 u1 = urand(p, s, move, slot(kKindMove, 0, 0, 1));
      const double2 u2 = urand(p, s, move, slot(kKindMove, 0, 0, 2));
      const double ptot = S.p_translation + S.p_swap;
      sh.kind = (u0.x * ptot < S.p_translation) ? 0 : (u0.y < 0.5 ? 2 : 3);
      sh.m = min(sh.n - 1, static_cast<int>(u1.x * sh.n));
      sh.axis = min(2, static_cast<int>(3.0 * u1.y));
      sh.disp = S.max_translation * 2.0 * (u2.x - 0.5);
      sh.u_acc = u2.y;
      sh.accept = 0;
    }
    __syncthreads();
    const int kind = sh.kind, n = sh.n, m = sh.m;
    const int nmb = n * nb;
    if (kind == 0 && n > 0)
    {
      // translation (translation.cpp:30-200): one Cartesian direction, uniform displacement
      if (tid < nb)
      {
        const double3 o = d3(pos[3 * (m * nb + tid)], pos[3 * (m * nb + tid) + 1], pos[3 * (m * nb + tid) + 2]);
        double3 nw = o;
        if (sh.axis == 0) nw.x += sh.disp;
        if (sh.axis == 1) nw.y += sh.disp;
        if (sh.axis == 2) nw.z += sh.disp;
        sh.old[tid] = nw;
        sh.bead[tid] = toFixed(S, nw, S.types[tid]);
        const int4 q = molS[m * nb + tid];
        sh.bead[nb + tid] = make_int4(q.x, q.y, q.z, S.types[tid]);
      }
      __syncthreads();
      evalBeads(sh, p, S, fwS, nfw, molS, nmb, 2 * nb, m, cl, eval);
      if (tid == 0)
      {
        const unsigned newMask = (1u << nb) - 1u;
        if (!(sh.ovl & newMask))
        {
          double dU = 0.0;
          for (int b = 0; b < nb; ++b) dU += (sh.efw[b] + sh.emm[b]) - (sh.efw[nb + b] + sh.emm[nb + b]);
          if (sh.u_acc < exp(-S.beta * dU))
          {
            sh.accept = 1;
            sh.energy += dU;
          }
        }
      }
      __syncthreads();
      if (sh.accept && tid < nb)
      {
        const int i = m * nb + tid;
        pos[3 * i] = sh.old[tid].x;
        pos[3 * i + 1] = sh.old[tid].y;
        pos[3 * i + 2] = sh.old[tid].z;
        const int4 q = sh.bead[tid];
        molS[i] = make_int4(q.x, q.y, q.z, S.types[tid] | (m << 8));
      }
    }
    else if (kind == 2 && n < S.max_molecules)
    {
      // CBMC insertion (insertion_cbmc.cpp:34-207): Pacc = beta f V / (N+1) W / W_IG
      growChain(sh, p, S, s, move, false, -1, fwS, nfw, molS, nmb, cl, eval);
      if (tid == 0 && !sh.fail)
      {
        const double pacc = S.beta * S.fugacity * S.volume / static_cast<double>(n + 1) * sh.W / S.w_ig;
        if (sh.u_acc < pacc)
        {
          sh.accept = 1;
          sh.energy += sh.eext + internalEnergy(p, S, sh.x);
        }
      }
      __syncthreads();
      if (sh.accept && tid < nb)
      {
        const int i = n * nb + tid;
        pos[3 * i] = sh.x[tid].x;
        pos[3 * i + 1] = sh.x[tid].y;
        pos[3 * i + 2] = sh.x[tid].z;
        molS[i] = toFixed(S, sh.x[tid], S.types[tid] | (n << 8));
      }
      if (tid == 0 && sh.accept) sh.n = n + 1;
    }
    else if (kind == 3 && n > 0)
    {
      // CBMC deletion (deletion_cbmc.cpp:34-195): Pacc = N / (beta f V) W_IG / W
      if (tid < nb)
      {
        const int i = m * nb + tid;
        sh.old[tid] = d3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
      }
      __syncthreads();
      growChain(sh, p, S, s, move, true, m, fwS, nfw, molS, nmb, cl, eval);
      if (tid == 0 && !sh.fail)
      {
        const double pacc = static_cast<double>(n) / (S.beta * S.fugacity * S.volume) * S.w_ig / sh.W;
        if (sh.u_acc < pacc)
        {
          sh.accept = 1;
          sh.energy -= sh.eext + internalEnergy(p, S, sh.old);
        }
      }
      __syncthreads();
      if (sh.accept && tid < nb && m != n - 1)
      {
        const int i = m * nb + tid, l = (n - 1) * nb + tid;
        pos[3 * i] = pos[3 * l];
        pos[3 * i + 1] = pos[3 * l + 1];
        pos[3 * i + 2] = pos[3 * l + 2];
        const int4 q = molS[l];
        molS[i] = make_int4(q.x, q.y, q.z, S.types[tid] | (m << 8));
      }
      if (tid == 0 && sh.accept) sh.n = n - 1;
    }
    __syncthreads();
    if (tid == 0 && record)
    {
      const int nn = sh.n;
      sh.stats[kind] += 1.0;
      sh.stats[4 + kind] += sh.accept ? 1.0 : 0.0;
      sh.stats[8] += nn;
      sh.stats[9] += static_cast<double>(nn) * nn;
      sh.stats[10] += sh.energy;
      sh.stats[11] += 1.0;
      const long long b = block_len > 0 ? static_cast<long long>(sh.stats[11] - 1.0) / block_len : 0;
      if (b < 5) sh.stats[12 + b] += nn;
    }
    __syncthreads();
  }
  if (tid == 0 && sh.pairs) atomicAdd(p.pairs + s, sh.pairs);
  if (rank == 0 && tid == 0)
  {
    p.n_mol[s] = sh.n;
    p.energy[s] = sh.energy;
    p.move_base[s] = move0 + moves;
    for (int k = 0; k < kStats; ++k) st[k] = sh.stats[k];
  }
  // no CTA leaves while another may still read its shared memory
  if (C > 1) cluster.sync();
}

// External energies of given beads in one system (single CTA).
__global__ void __launch_bounds__(128) beadKernel(Params p, int s, int fw_cap, const double* xyz, const int* types,
                                                  int nbd, int skip, double* out_fw, double* out_mm, int* out_ovl)
{
  extern __shared__ __align__(16) unsigned char smem[];
  Shared& sh = *reinterpret_cast<Shared*>(smem);
  int4* fwS = dynamicBase(smem);
  int4* molS = fwS + fw_cap;
  const Cl cl{0, 1};
  const SysDev& S = p.sys[s];
  const int tid = threadIdx.x;
  for (int i = tid; i < S.n_fw; i += blockDim.x) fwS[i] = p.fw[S.fw_offset + i];
  for (int i = tid; i < kMaxTypes * kMaxTypes; i += blockDim.x) sh.tab[i] = p.ljf[i];
  const double* pos = p.pos + 3ll * S.pos_offset;
  const int n = p.n_mol[s], nb = S.nb;
  for (int i = tid; i < n * nb; i += blockDim.x)
  {
    const int m = i / nb, b = i - m * nb;
    molS[i] = toFixed(S, d3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), S.types[b] | (m << 8));
  }
  if (tid < nbd) sh.bead[tid] = toFixed(S, d3(xyz[3 * tid], xyz[3 * tid + 1], xyz[3 * tid + 2]), types[tid]);
  if (tid == 0) sh.pairs = 0ull;
  __syncthreads();
  int eval = 0;
  evalBeads(sh, p, S, fwS, S.n_fw, molS, n * nb, nbd, skip, cl, eval);
  if (tid < nbd)
  {
    out_fw[tid] = sh.efw[tid];
    out_mm[tid] = sh.emm[tid];
    out_ovl[tid] = (sh.ovl >> tid) & 1u;
  }
}

// Growth in vacuum: chains grown one per CTA at a time, n chains in total.
__global__ void __launch_bounds__(128) vacuumKernel(Params p, long long n, double* w, double* theta, double* cphi)
{
  extern __shared__ __align__(16) unsigned char smem[];
  Shared& sh = *reinterpret_cast<Shared*>(smem);
  const Cl cl{0, 1};
  const SysDev& S = p.sys[0];
  const int tid = threadIdx.x, nb = S.nb;
  for (int i = tid; i < kMaxTypes * kMaxTypes; i += blockDim.x) sh.tab[i] = p.ljf[i];
  if (tid == 0) sh.pairs = 0ull;
  int eval = 0;
  __syncthreads();
  for (long long c = blockIdx.x; c < n; c += gridDim.x)
  {
    growChain(sh, p, S, 0, c, false, -1, nullptr, 0, nullptr, 0, cl, eval);
    if (tid == 0)
    {
      w[c] = sh.fail ? 0.0 : sh.W;
      for (int j = 2; theta && j < nb; ++j)
      {
        const double3 ab = sub(sh.x[j - 2], sh.x[j - 1]), cb = sub(sh.x[j], sh.x[j - 1]);
        theta[c * (nb - 2) + j - 2] = atan2(sqrt(dot(cross(ab, cb), cross(ab, cb))), dot(ab, cb));
      }
      for (int j = 3; cphi && j < nb; ++j)
      {
        const double3 dab = sub(sh.x[j - 3], sh.x[j - 2]), dcb = normalized(sub(sh.x[j - 1], sh.x[j - 2]));
        const double3 ddc = sub(sh.x[j], sh.x[j - 1]);
        const double3 dr = normalized(sub(dab, scale(dot(dab, dcb), dcb)));
        const double3 ds = normalized(sub(ddc, scale(dot(ddc, dcb), dcb)));
        cphi[c * (nb - 3) + j - 3] = dot(dr, ds);
      }
    }
    __syncthreads();
  }
}
}  // namespace

struct rg_alkane
{
  rg_ctx* ctx = nullptr;
  int n_systems = 0;
  Params p{};
  std::vector<SysDev> sys;
  std::vector<int> order;  // systems by decreasing work
  int* d_order = nullptr;
  int4* d_fw = nullptr;
  SysDev* d_sys = nullptr;
  Ctrl* d_ctrl = nullptr;
  float4* d_ljf = nullptr;
  double2* d_ljd = nullptr;
  long long block_len = 0;
  size_t pos_doubles = 0;
  rg_alkane_plan plan{};
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_moves = 0;
  int graph_kernels = 0;
  int64_t launches = 0;  // Monte Carlo kernel launches enqueued (graph kernel nodes included)
  int max_smem = 0;
};

namespace
{
size_t sharedBytes(int fw_cap, int mol_cap)
{
  return ((sizeof(Shared) + 15) & ~static_cast<size_t>(15)) + sizeof(int4) * static_cast<size_t>(fw_cap + mol_cap);
}

// capacities of the class [b, e) of the work order with cluster size C
void classCaps(const rg_alkane* a, int b, int e, int C, int* fw_cap, int* mol_cap)
{
  int f = 0, mc = 0;
  for (int k = b; k < e; ++k)
  {
    const SysDev& S = a->sys[a->order[k]];
    f = std::max(f, (S.n_fw + C - 1) / C);
    mc = std::max(mc, S.max_molecules * S.nb);
  }
  *fw_cap = f;
  *mol_cap = mc;
}

// Whether clusters of C CTAs of T threads with `smem` bytes each can be resident at all on this device.
template <int T>
bool clusterFits(int C, size_t smem)
{
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(C));
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(C);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveClusters(&n, alkaneKernel<T>, &cfg);
  if (e != cudaSuccess)
  {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}

bool planFits(const rg_alkane* a, const rg_alkane_plan& pl)
{
  const int split = std::min(std::max(pl.split, 0), a->n_systems);
  const int cls[2][3] = {{0, split, pl.cluster_big}, {split, a->n_systems, pl.cluster_small}};
  for (auto& c : cls)
  {
    if (c[0] >= c[1]) continue;
    int f, m;
    classCaps(a, c[0], c[1], c[2], &f, &m);
    const size_t smem = sharedBytes(f, m);
    if (smem > static_cast<size_t>(a->max_smem)) return false;
    const bool fits = pl.threads == 512   ? clusterFits<512>(c[2], smem)
                      : pl.threads == 256 ? clusterFits<256>(c[2], smem)
                                          : clusterFits<128>(c[2], smem);
    if (!fits) return false;
  }
  return true;
}

template <int T>
cudaError_t launchClass(rg_alkane* a, cudaStream_t stream, int b, int e, int C, int moves)
{
  if (b >= e) return cudaSuccess;
  int fw_cap, mol_cap;
  classCaps(a, b, e, C, &fw_cap, &mol_cap);
  const size_t smem = sharedBytes(fw_cap, mol_cap);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>((e - b) * C));
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = static_cast<unsigned>(C);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, alkaneKernel<T>, a->p, static_cast<const int*>(a->d_order + b), fw_cap, moves);
}

cudaError_t launchPlan(rg_alkane* a, const rg_alkane_plan& pl, int moves, bool count = true)
{
  const int split = std::min(std::max(pl.split, 0), a->n_systems);
  if (count) a->launches += (split > 0 ? 1 : 0) + (split < a->n_systems ? 1 : 0);
  cudaStream_t main = a->ctx->stream;
  cudaError_t err = cudaEventRecord(a->fork, main);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(a->side, a->fork, 0);
  auto go = [&](cudaStream_t st, int b, int e, int C) {
    return pl.threads == 512   ? launchClass<512>(a, st, b, e, C, moves)
           : pl.threads == 256 ? launchClass<256>(a, st, b, e, C, moves)
                               : launchClass<128>(a, st, b, e, C, moves);
  };
  if (err == cudaSuccess) err = go(main, 0, split, pl.cluster_big);
  if (err == cudaSuccess) err = go(a->side, split, a->n_systems, pl.cluster_small);
  if (err == cudaSuccess) err = cudaEventRecord(a->join, a->side);
  if (err == cudaSuccess) err = cudaStreamWaitEvent(main, a->join, 0);
  return err;
}

rg_status rebuildGraph(rg_alkane* a)
{
  rg_ctx* ctx = a->ctx;
  if (a->graph)
  {
    cudaGraphExecDestroy(a->graph);
    a->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  RG_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const cudaError_t le = launchPlan(a, a->plan, a->plan.moves_per_launch, false);
  const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
  if (le != cudaSuccess) return rg::cudaFail(ctx, le, "alkane graph capture");
  if (ce != cudaSuccess) return rg::cudaFail(ctx, ce, "cudaStreamEndCapture");
  const cudaError_t ie = cudaGraphInstantiate(&a->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) return rg::cudaFail(ctx, ie, "cudaGraphInstantiate");
  a->graph_moves = a->plan.moves_per_launch;
  const int split = std::min(std::max(a->plan.split, 0), a->n_systems);
  a->graph_kernels = (split > 0 ? 1 : 0) + (split < a->n_systems ? 1 : 0);
  return RG_OK;
}

void freeAll(rg_alkane* a)
{
  if (a->graph) cudaGraphExecDestroy(a->graph);
  if (a->side) cudaStreamDestroy(a->side);
  if (a->fork) cudaEventDestroy(a->fork);
  if (a->join) cudaEventDestroy(a->join);
  cudaFree(a->d_order);
  cudaFree(a->d_fw);
  cudaFree(a->d_sys);
  cudaFree(a->d_ctrl);
  cudaFree(a->d_ljf);
  cudaFree(a->d_ljd);
  cudaFree(a->p.pos);
  cudaFree(a->p.n_mol);
  cudaFree(a->p.energy);
  cudaFree(a->p.move_base);
  cudaFree(a->p.stats);
  cudaFree(a->p.pairs);
}

rg_status fillTables(rg_ctx* ctx, const rg_forcefield* ff, std::vector<float4>& ljf, std::vector<double2>& ljd)
{
  if (ff->n_types < 1 || ff->n_types > kMaxTypes) return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_alkane: at most 16 types");
  ljf.assign(kMaxTypes * kMaxTypes, make_float4(0, 0, 0, 0));
  ljd.assign(kMaxTypes * kMaxTypes, make_double2(0, 1));
  for (int a = 0; a < ff->n_types; ++a)
    for (int b = 0; b < ff->n_types; ++b)
    {
      const int k = a * ff->n_types + b;
      if (!ff->lj[k]) continue;
      const double e4 = 4.0 * ff->epsilon[k], s2 = ff->sigma[k] * ff->sigma[k];
      ljf[a * kMaxTypes + b] = make_float4(static_cast<float>(e4), static_cast<float>(s2),
                                           static_cast<float>(ff->shift[k]), 0.0f);
      ljd[a * kMaxTypes + b] = make_double2(e4, s2);
    }
  return RG_OK;
}

rg_status validateChain(rg_ctx* ctx, const rg_alkane_chain& c, int n_types)
{
  if (c.n_beads < 2 || c.n_beads > kMaxBeads) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: n_beads in 2..8");
  if (c.n_first_bead_trials < 1 || c.n_first_bead_trials > kMaxTrials || c.n_trial_directions < 1 ||
      c.n_trial_directions > kMaxTrials || c.n_torsion_trials < 1 || c.n_torsion_trials > kMaxTorsion)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: trial counts out of range (16, 16, 128)");
  for (int b = 0; b < c.n_beads; ++b)
    if (c.types[b] < 0 || c.types[b] >= n_types) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: bead type");
  if (!(c.bond_length > 0.0) || !(c.bend_k > 0.0))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: needs a positive bond length and bend constant");
  return RG_OK;
}

SysDev makeSysDev(const rg_box& box, const rg_alkane_chain& c, double beta)
{
  SysDev S{};
  const rg::HostBox hb = rg::makeHostBox(&box);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      S.c[i][j] = hb.c[i][j];
      S.ic[i][j] = hb.ic[i][j];
      S.hf[i][j] = static_cast<float>(hb.c[i][j]);
    }
  S.triclinic = hb.triclinic ? 1 : 0;
  S.volume = hb.volume;
  S.beta = beta;
  S.nb = c.n_beads;
  S.n_first = c.n_first_bead_trials;
  S.n_dir = c.n_trial_directions;
  S.n_tors = c.n_torsion_trials;
  for (int b = 0; b < c.n_beads; ++b) S.types[b] = c.types[b];
  S.bond = c.bond_length;
  S.bend_k = c.bend_k;
  S.bend_theta0 = c.bend_theta0;
  S.sigma_theta = 1.0 / std::sqrt(beta * c.bend_k);
  for (int k = 0; k < 4; ++k) S.torsion[k] = c.torsion[k];
  return S;
}
}  // namespace

extern "C" rg_status rg_alkane_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_alkane_system* systems,
                                      int n_systems, uint64_t seed, rg_alkane** out)
{
  if (!ctx || !ff || !systems || !out || n_systems < 1) return RG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float4> ljf;
  std::vector<double2> ljd;
  rg_status st = fillTables(ctx, ff, ljf, ljd);
  if (st) return st;
  auto* a = new rg_alkane();
  a->ctx = ctx;
  a->n_systems = n_systems;
  std::vector<int4> fw;
  std::vector<double> work(n_systems);
  size_t pos_beads = 0;
  for (int s = 0; s < n_systems; ++s)
  {
    const rg_alkane_system& q = systems[s];
    st = validateChain(ctx, q.chain, ff->n_types);
    if (!st && (q.max_molecules < 1 || q.max_molecules > kMaxMolecules))
      st = rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: max_molecules in 1..256");
    if (!st && (q.n_framework < 0 || (q.n_framework > 0 && !q.framework)))
      st = rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: framework atoms");
    if (!st && !(q.beta > 0.0 && q.fugacity > 0.0 && q.w_ig > 0.0))
      st = rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: beta, fugacity and w_ig must be positive");
    if (st)
    {
      delete a;
      return st;
    }
    SysDev S = makeSysDev(q.box, q.chain, q.beta);
    S.fugacity = q.fugacity;
    S.w_ig = q.w_ig;
    S.max_translation = q.max_translation;
    S.p_translation = q.p_translation;
    S.p_swap = q.p_swap;
    S.max_molecules = q.max_molecules;
    S.pos_offset = static_cast<int>(pos_beads);
    pos_beads += static_cast<size_t>(q.max_molecules) * q.chain.n_beads;
    S.fw_offset = static_cast<int>(fw.size());
    // keep the framework atoms that interact with some bead type
    for (int i = 0; i < q.n_framework; ++i)
    {
      const rg_atom& at = q.framework[i];
      if (at.type >= ff->n_types)
      {
        delete a;
        return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane: framework atom type");
      }
      bool any = false;
      for (int b = 0; b < q.chain.n_beads; ++b) any |= ff->lj[at.type * ff->n_types + q.chain.types[b]] != 0 &&
                                                      ff->epsilon[at.type * ff->n_types + q.chain.types[b]] != 0.0;
      if (!any) continue;
      const double s0 = S.ic[0][0] * at.x + S.ic[1][0] * at.y + S.ic[2][0] * at.z;
      const double s1 = S.ic[0][1] * at.x + S.ic[1][1] * at.y + S.ic[2][1] * at.z;
      const double s2 = S.ic[0][2] * at.x + S.ic[1][2] * at.y + S.ic[2][2] * at.z;
      auto fx = [](double v) {
        v -= std::floor(v);
        return static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(v * 4294967296.0)));
      };
      fw.push_back(make_int4(fx(s0), fx(s1), fx(s2), static_cast<int>(at.type)));
    }
    S.n_fw = static_cast<int>(fw.size()) - S.fw_offset;
    work[s] = static_cast<double>(S.n_fw + 64) *
              (S.n_first + (S.nb - 1) * S.n_dir + 0.5 * S.nb);
    a->sys.push_back(S);
  }
  a->order.resize(n_systems);
  std::iota(a->order.begin(), a->order.end(), 0);
  std::stable_sort(a->order.begin(), a->order.end(), [&](int x, int y) { return work[x] > work[y]; });
  a->pos_doubles = 3 * pos_beads;
  a->p.seed = seed;
  a->p.rc2_fw = static_cast<float>(ff->cutoff_framework_vdw * ff->cutoff_framework_vdw);
  a->p.rc2_mm = static_cast<float>(ff->cutoff_molecule_vdw * ff->cutoff_molecule_vdw);
  a->p.overlap_f = static_cast<float>(ff->overlap_criteria);
  cudaError_t err = cudaDeviceGetAttribute(&a->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  auto alloc = [&](void** ptr, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
  };
  alloc(reinterpret_cast<void**>(&a->d_order), sizeof(int) * n_systems);
  alloc(reinterpret_cast<void**>(&a->d_fw), sizeof(int4) * fw.size());
  alloc(reinterpret_cast<void**>(&a->d_sys), sizeof(SysDev) * n_systems);
  alloc(reinterpret_cast<void**>(&a->d_ctrl), sizeof(Ctrl));
  alloc(reinterpret_cast<void**>(&a->d_ljf), sizeof(float4) * ljf.size());
  alloc(reinterpret_cast<void**>(&a->d_ljd), sizeof(double2) * ljd.size());
  alloc(reinterpret_cast<void**>(&a->p.pos), sizeof(double) * a->pos_doubles);
  alloc(reinterpret_cast<void**>(&a->p.n_mol), sizeof(int) * n_systems);
  alloc(reinterpret_cast<void**>(&a->p.energy), sizeof(double) * n_systems);
  alloc(reinterpret_cast<void**>(&a->p.move_base), sizeof(long long) * n_systems);
  alloc(reinterpret_cast<void**>(&a->p.stats), sizeof(double) * kStats * n_systems);
  alloc(reinterpret_cast<void**>(&a->p.pairs), sizeof(unsigned long long) * n_systems);
  cudaStream_t sm = ctx->stream;
  Ctrl ctrl{0, 0, 0};
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a->d_order, a->order.data(), sizeof(int) * n_systems, cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess && !fw.empty())
    err = cudaMemcpyAsync(a->d_fw, fw.data(), sizeof(int4) * fw.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a->d_sys, a->sys.data(), sizeof(SysDev) * n_systems, cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(a->d_ctrl, &ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a->d_ljf, ljf.data(), sizeof(float4) * ljf.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(a->d_ljd, ljd.data(), sizeof(double2) * ljd.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.pos, 0, sizeof(double) * std::max<size_t>(a->pos_doubles, 2), sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.n_mol, 0, sizeof(int) * n_systems, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.energy, 0, sizeof(double) * n_systems, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.move_base, 0, sizeof(long long) * n_systems, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.stats, 0, sizeof(double) * kStats * n_systems, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(a->p.pairs, 0, sizeof(unsigned long long) * n_systems, sm);
  if (err == cudaSuccess) err = cudaStreamSynchronize(sm);
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(alkaneKernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, a->max_smem);
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(alkaneKernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, a->max_smem);
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(alkaneKernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, a->max_smem);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&a->join, cudaEventDisableTiming);
  if (err != cudaSuccess)
  {
    freeAll(a);
    delete a;
    return rg::cudaFail(ctx, err, "rg_alkane_create");
  }
  a->p.sys = a->d_sys;
  a->p.fw = a->d_fw;
  a->p.ctrl = a->d_ctrl;
  a->p.ljf = a->d_ljf;
  a->p.ljd = a->d_ljd;
  // default plan: one CTA per system, 128 threads, 500 moves per launch (a launch lasts as long as its slowest system,
  // so longer launches average the systems' move-to-move spread: 1.69e6 moves/s at 64 per launch, 1.79e6 at 256-1000
  // on the 64-system batch)
  a->plan = rg_alkane_plan{1, 1, 128, 0, 500, 0, 0.0};
  if (!planFits(a, a->plan))
  {
    a->plan.cluster_big = a->plan.cluster_small = 4;
    if (!planFits(a, a->plan))
    {
      freeAll(a);
      delete a;
      return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_alkane: a system does not fit in shared memory");
    }
  }
  st = rebuildGraph(a);
  if (st)
  {
    freeAll(a);
    delete a;
    return st;
  }
  *out = a;
  return RG_OK;
}

extern "C" rg_status rg_alkane_destroy(rg_alkane* a)
{
  if (!a) return RG_OK;
  cudaSetDevice(a->ctx->device);
  cudaStreamSynchronize(a->ctx->stream);
  freeAll(a);
  delete a;
  return RG_OK;
}

extern "C" rg_status rg_alkane_set_plan(rg_alkane* a, const rg_alkane_plan* plan)
{
  if (!a || !plan) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  const int okC[3] = {1, 2, 4};
  auto validC = [&](int c) { return std::find(okC, okC + 3, c) != okC + 3; };
  if (!validC(plan->cluster_big) || !validC(plan->cluster_small) ||
      (plan->threads != 128 && plan->threads != 256 && plan->threads != 512) ||
      plan->moves_per_launch < 1 || plan->split < 0 || plan->split > a->n_systems)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane_set_plan: clusters 1/2/4, threads 128/256/512");
  if (!planFits(a, *plan)) return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_alkane_set_plan: exceeds shared memory");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  a->plan = *plan;
  return rebuildGraph(a);
}

extern "C" rg_status rg_alkane_get_plan(rg_alkane* a, rg_alkane_plan* plan)
{
  if (!a || !plan) return RG_ERR_INVALID_ARGUMENT;
  *plan = a->plan;
  return RG_OK;
}

extern "C" rg_status rg_alkane_run(rg_alkane* a, int64_t moves, int record)
{
  if (!a || moves < 0) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (record && a->block_len == 0) a->block_len = moves / 5 > 0 ? moves / 5 : 1;
  Ctrl c{record ? 1 : 0, 0, a->block_len};
  RG_CUDA(ctx, cudaMemcpyAsync(a->d_ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, ctx->stream));
  int64_t left = moves;
  while (left >= a->graph_moves)
  {
    RG_CUDA(ctx, cudaGraphLaunch(a->graph, ctx->stream));
    a->launches += a->graph_kernels;
    left -= a->graph_moves;
  }
  // (the control block is copied from pageable memory: staged before cudaMemcpyAsync returns)
  if (left > 0) RG_CUDA(ctx, launchPlan(a, a->plan, static_cast<int>(left)));
  return RG_OK;
}

extern "C" rg_status rg_alkane_autotune(rg_alkane* a, int moves_per_candidate, rg_alkane_plan* chosen)
{
  if (!a || moves_per_candidate < 1) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int n = a->n_systems;
  // snapshot of the state: every candidate starts from it, and it is restored at the end
  double *pos = nullptr, *energy = nullptr, *stats = nullptr;
  int* nm = nullptr;
  long long* mb = nullptr;
  unsigned long long* pc = nullptr;
  cudaError_t err = cudaMalloc(&pos, sizeof(double) * std::max<size_t>(a->pos_doubles, 2));
  if (err == cudaSuccess) err = cudaMalloc(&pc, sizeof(unsigned long long) * n);
  if (err == cudaSuccess) err = cudaMalloc(&energy, sizeof(double) * n);
  if (err == cudaSuccess) err = cudaMalloc(&stats, sizeof(double) * kStats * n);
  if (err == cudaSuccess) err = cudaMalloc(&nm, sizeof(int) * n);
  if (err == cudaSuccess) err = cudaMalloc(&mb, sizeof(long long) * n);
  cudaStream_t sm = ctx->stream;
  auto copyState = [&](bool save) {
    auto cp = [&](void* x, void* y, size_t b) {
      if (err == cudaSuccess) err = cudaMemcpyAsync(save ? x : y, save ? y : x, b, cudaMemcpyDeviceToDevice, sm);
    };
    cp(pos, a->p.pos, sizeof(double) * a->pos_doubles);
    cp(energy, a->p.energy, sizeof(double) * n);
    cp(stats, a->p.stats, sizeof(double) * kStats * n);
    cp(nm, a->p.n_mol, sizeof(int) * n);
    cp(mb, a->p.move_base, sizeof(long long) * n);
    cp(pc, a->p.pairs, sizeof(unsigned long long) * n);
  };
  copyState(true);
  Ctrl c{0, 0, a->block_len};
  if (err == cudaSuccess) err = cudaMemcpyAsync(a->d_ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, sm);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (err == cudaSuccess) err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  std::vector<rg_alkane_plan> cands;
  const int quarter = std::max(1, n / 4), half = std::max(1, n / 2);
  const int combos[][3] = {{1, 1, 0}, {2, 2, 0}, {4, 4, 0}, {2, 1, 0}, {2, 1, 1}, {4, 1, 0}, {4, 2, 0}, {4, 2, 1}};
  for (int t : {128, 256, 512})
    for (auto& cb : combos)
    {
      rg_alkane_plan pl{cb[0], cb[1], t, cb[0] == cb[1] ? n : (cb[2] ? half : quarter), a->plan.moves_per_launch, 0,
                        0.0};
      if (planFits(a, pl)) cands.push_back(pl);
    }
  float best = 1e30f;
  rg_alkane_plan bestPlan = a->plan;
  for (rg_alkane_plan& pl : cands)
  {
    copyState(false);
    // one untimed warm-up launch, then the timed ones
    if (err == cudaSuccess) err = launchPlan(a, pl, 1);
    copyState(false);
    if (err == cudaSuccess) err = cudaEventRecord(e0, sm);
    if (err == cudaSuccess) err = launchPlan(a, pl, moves_per_candidate);
    if (err == cudaSuccess) err = cudaEventRecord(e1, sm);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (err != cudaSuccess) break;
    pl.ms_per_move = ms / moves_per_candidate;
    if (ms < best)
    {
      best = ms;
      bestPlan = pl;
    }
  }
  copyState(false);
  if (err == cudaSuccess) err = cudaStreamSynchronize(sm);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(pos);
  cudaFree(energy);
  cudaFree(stats);
  cudaFree(nm);
  cudaFree(mb);
  cudaFree(pc);
  if (err != cudaSuccess) return rg::cudaFail(ctx, err, "rg_alkane_autotune");
  a->plan = bestPlan;
  const rg_status st = rebuildGraph(a);
  if (st) return st;
  if (chosen) *chosen = bestPlan;
  return RG_OK;
}

extern "C" rg_status rg_alkane_results(rg_alkane* a, rg_gcmc_chain_result* out)
{
  if (!a || !out) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int n = a->n_systems;
  std::vector<int> nm(n);
  std::vector<double> e(n), s(static_cast<size_t>(kStats) * n);
  RG_CUDA(ctx, cudaMemcpyAsync(nm.data(), a->p.n_mol, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(e.data(), a->p.energy, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(s.data(), a->p.stats, sizeof(double) * s.size(), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < n; ++c)
  {
    rg_gcmc_chain_result& r = out[c];
    std::memset(&r, 0, sizeof(r));
    const double* q = &s[static_cast<size_t>(c) * kStats];
    r.n_molecules = nm[c];
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
    for (int b = 0; b < 5; ++b) r.block_n[b] = a->block_len > 0 ? q[12 + b] / static_cast<double>(a->block_len) : 0.0;
  }
  return RG_OK;
}

extern "C" rg_status rg_alkane_get_positions(rg_alkane* a, int system, double* xyz, int capacity_doubles,
                                             int* n_molecules)
{
  if (!a || !xyz || !n_molecules || system < 0 || system >= a->n_systems) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  int n = 0;
  RG_CUDA(ctx, cudaMemcpyAsync(&n, a->p.n_mol + system, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const SysDev& S = a->sys[system];
  const int need = 3 * n * S.nb;
  if (need > capacity_doubles) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane_get_positions: capacity");
  if (need > 0)
    RG_CUDA(ctx, cudaMemcpyAsync(xyz, a->p.pos + 3ll * S.pos_offset, sizeof(double) * need, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *n_molecules = n;
  return RG_OK;
}

extern "C" rg_status rg_alkane_set_positions(rg_alkane* a, int system, const double* xyz, int n_molecules,
                                             double energy)
{
  if (!a || system < 0 || system >= a->n_systems || n_molecules < 0 || (n_molecules > 0 && !xyz))
    return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  const SysDev& S = a->sys[system];
  if (n_molecules > S.max_molecules) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_alkane_set_positions: count");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n_molecules > 0)
    RG_CUDA(ctx, cudaMemcpyAsync(a->p.pos + 3ll * S.pos_offset, xyz, sizeof(double) * 3 * n_molecules * S.nb,
                                 cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(a->p.n_mol + system, &n_molecules, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(a->p.energy + system, &energy, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

extern "C" rg_status rg_alkane_bead_energies(rg_alkane* a, int system, const double* xyz_beads, const int32_t* types,
                                             int n_beads, int skip, double* fw, double* mm, int32_t* overlap)
{
  if (!a || !xyz_beads || !types || !fw || !mm || !overlap || system < 0 || system >= a->n_systems || n_beads < 1 ||
      n_beads > kMaxTrials)
    return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const SysDev& S = a->sys[system];
  const size_t smem = sharedBytes(S.n_fw, S.max_molecules * S.nb);
  if (smem > static_cast<size_t>(a->max_smem))
    return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_alkane_bead_energies: system exceeds one CTA's shared memory");
  for (int b = 0; b < n_beads; ++b)
    if (types[b] < 0 || types[b] >= kMaxTypes) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "bead type");
  // staging: xyz (48 doubles), types (16), fw (16), mm (16), overlap (16)
  void* d = nullptr;
  rg_status st = rg::scratch(ctx, 0, 256 * sizeof(double), &d);
  if (st) return st;
  double* dx = static_cast<double*>(d);
  int* dt = reinterpret_cast<int*>(dx + 48);
  double* dfw = dx + 64;
  double* dmm = dx + 80;
  int* dov = reinterpret_cast<int*>(dx + 96);
  RG_CUDA(ctx, cudaMemcpyAsync(dx, xyz_beads, sizeof(double) * 3 * n_beads, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(dt, types, sizeof(int) * n_beads, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaFuncSetAttribute(beadKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  beadKernel<<<1, 128, smem, ctx->stream>>>(a->p, system, S.n_fw, dx, dt, n_beads, skip, dfw, dmm, dov);
  RG_CUDA(ctx, cudaGetLastError());
  RG_CUDA(ctx, cudaMemcpyAsync(fw, dfw, sizeof(double) * n_beads, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(mm, dmm, sizeof(double) * n_beads, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(overlap, dov, sizeof(int) * n_beads, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

extern "C" rg_status rg_alkane_grow_vacuum(rg_ctx* ctx, const rg_forcefield* ff, const rg_alkane_chain* chain,
                                           double beta, int64_t n, uint64_t seed, double* w_mean, double* w,
                                           double* theta, double* cos_phi)
{
  if (!ctx || !ff || !chain || n < 1 || !(beta > 0.0)) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_status st = validateChain(ctx, *chain, ff->n_types);
  if (st) return st;
  std::vector<float4> ljf;
  std::vector<double2> ljd;
  st = fillTables(ctx, ff, ljf, ljd);
  if (st) return st;
  rg_box box{};
  box.cell[0] = box.cell[4] = box.cell[8] = 100.0;
  SysDev S = makeSysDev(box, *chain, beta);
  S.fugacity = 1.0;
  S.w_ig = 1.0;
  const int nb = chain->n_beads;
  const size_t bytes = sizeof(SysDev) + sizeof(float4) * ljf.size() + sizeof(double2) * ljd.size() +
                       sizeof(double) * n * (1 + std::max(0, nb - 2) + std::max(0, nb - 3)) + 256;
  void* d = nullptr;
  st = rg::scratch(ctx, 1, bytes, &d);
  if (st) return st;
  unsigned char* q = static_cast<unsigned char*>(d);
  SysDev* dS = reinterpret_cast<SysDev*>(q);
  float4* dljf = reinterpret_cast<float4*>(q + ((sizeof(SysDev) + 15) & ~size_t(15)));
  double2* dljd = reinterpret_cast<double2*>(dljf + ljf.size());
  double* dw = reinterpret_cast<double*>(dljd + ljd.size());
  double* dth = dw + n;
  double* dcp = dth + n * std::max(0, nb - 2);
  RG_CUDA(ctx, cudaMemcpyAsync(dS, &S, sizeof(SysDev), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(dljf, ljf.data(), sizeof(float4) * ljf.size(), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(dljd, ljd.data(), sizeof(double2) * ljd.size(), cudaMemcpyHostToDevice, ctx->stream));
  Params p{};
  p.sys = dS;
  p.ljf = dljf;
  p.ljd = dljd;
  p.rc2_fw = p.rc2_mm = 0.0f;
  p.overlap_f = static_cast<float>(ff->overlap_criteria);
  p.seed = seed;
  const size_t smem = sharedBytes(0, 0);
  RG_CUDA(ctx, cudaFuncSetAttribute(vacuumKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int sms = 0;
  RG_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const long long blocks = std::min<long long>(n, 8ll * sms);
  vacuumKernel<<<static_cast<unsigned>(blocks), 128, smem, ctx->stream>>>(p, n, dw, nb > 2 ? dth : nullptr,
                                                                         nb > 3 ? dcp : nullptr);
  RG_CUDA(ctx, cudaGetLastError());
  std::vector<double> hw(n);
  RG_CUDA(ctx, cudaMemcpyAsync(hw.data(), dw, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  if (theta && nb > 2)
    RG_CUDA(ctx, cudaMemcpyAsync(theta, dth, sizeof(double) * n * (nb - 2), cudaMemcpyDeviceToHost, ctx->stream));
  if (cos_phi && nb > 3)
    RG_CUDA(ctx, cudaMemcpyAsync(cos_phi, dcp, sizeof(double) * n * (nb - 3), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  double sum = 0.0;
  for (double v : hw) sum += v;
  if (w) std::memcpy(w, hw.data(), sizeof(double) * n);
  if (w_mean) *w_mean = sum / static_cast<double>(n);
  return RG_OK;
}

extern "C" rg_status rg_alkane_launch_count(rg_alkane* a, int64_t* launches)
{
  if (!a || !launches) return RG_ERR_INVALID_ARGUMENT;
  *launches = a->launches;
  return RG_OK;
}

extern "C" rg_status rg_alkane_pair_count(rg_alkane* a, uint64_t* total)
{
  if (!a || !total) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = a->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<unsigned long long> v(a->n_systems);
  RG_CUDA(ctx, cudaMemcpyAsync(v.data(), a->p.pairs, sizeof(unsigned long long) * v.size(), cudaMemcpyDeviceToHost,
                               ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  unsigned long long t = 0;
  for (unsigned long long x : v) t += x;
  *total = t;
  return RG_OK;
}

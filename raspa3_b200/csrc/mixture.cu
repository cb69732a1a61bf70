// Monte Carlo of one large system of several rigid components on the whole GPU (rg_mixture_*).
//
// A single system (tens of thousands of atoms, thousands of k-vectors) has too little work per move for one CTA and
// too much for a CPU core, so every move runs on all SMs: a cooperative persistent kernel of one CTA per SM.
//  * The molecule sites are split into contiguous slices, one per CTA; the k-vectors into ranges, one per CTA. Each
//    CTA keeps its range of the structure factors S(k) and the structure-factor changes of the move's candidates in
//    shared memory, and updates its range on acceptance: S(k) never crosses the GPU.
//  * A phase evaluates a set of trial atoms (framework energy from the tricubic grids, molecule-molecule Lennard-Jones
//    and real-space Ewald over the CTA's slice in FP32 from exact fixed-point displacements, accumulated in FP64) and
//    a set of Ewald candidates (energy change over the CTA's k-range, FP64). Each CTA writes one row of partial sums;
//    after a grid barrier every CTA adds the rows in CTA order, so every CTA holds identical totals, draws the same
//    counter-based random numbers and takes the same decision: nothing else is exchanged, and every CTA applies the
//    (identical) updates of positions and molecule lists itself. Every value such an update reads is read before the
//    phase's barrier, when no CTA can have started writing it.
//  * Moves with all trial positions known up front need one phase: translation, rotation, CBMC deletion (the retrace
//    orientations sit on the old first bead) and identity change (the new first bead sits on the old one). A CBMC
//    insertion needs two (first bead, then orientations).
//  * The grid barrier is this file's own: a generation counter in global memory, spin-waits bounded by an iteration
//    limit after which an error flag is raised and every CTA leaves; the host reports RG_ERR_TIMEOUT.
// Reference moves (file:line in the RASPA3 tree): mc_moves/component/translation.cpp:30-200, rotation.cpp:30-190,
// insertion_cbmc.cpp:34-207, deletion_cbmc.cpp:34-195, identity_change.cpp:33-290 with
// cbmc/multiple_first_bead.cpp:20-76, 136-168; energies cbmc/interactions_framework_molecule.cpp,
// cbmc/interactions_intermolecular.cpp, interactions/ewald.cpp:1043-1244 (Fourier difference) and :1164-1238 (self
// and exclusion terms of inserted / deleted rigid molecules, constant per component).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"
#include "fastmath.cuh"
#include "rng.cuh"

namespace
{
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxComp = 4;
constexpr int kMaxAtoms = 4;
constexpr int kMaxTrials = 12;
constexpr int kMaxItems = 96;          // trial atoms of one phase
constexpr int kMaxCand = kMaxTrials;   // Ewald candidates of one phase
constexpr int kMaxCandAtoms = 2 * kMaxAtoms;
constexpr int kSegLen = 4;        // k-vectors per segment of the candidates' Ewald sums (one (kx, ky) per segment)
constexpr int kMaxCells = 1024;   // cells of the pair loop's binning of a CTA's slice
constexpr int kPairWarps = kWarps - 1;  // warps of the pair loop (the last one interpolates the grids meanwhile)
static_assert(kMaxCand <= 2 * kWarps, "two candidates per warp in the energy sums");
constexpr int kMaxTypes = 16;
constexpr int kRow = kMaxItems + kMaxCand + 4;  // columns of partial sums per CTA (last 4: overlap-bit words)
constexpr int kMaxBlocks = 256;                 // CTAs of the cooperative launch (lanes x 8 in the column sums)
constexpr int kFwSlice = 512;                   // framework atoms of a CTA's slice kept in shared memory
constexpr long long kSpinLimit = 1ll << 22;
constexpr int kStats = 24;
constexpr float kFix = 2.3283064365386963e-10f;  // 2^-32

struct Comp
{
  int n_atoms, starting_bead;
  int types[kMaxAtoms];
  double charges[kMaxAtoms], masses[kMaxAtoms], offsets[kMaxAtoms][3];
  double fugacity, w_ig, self_excl;
  const double* vdw_grid[kMaxAtoms];
  // learned first-bead proposal (null: uniform)
  const double* prop_cdf;
  const double* prop_q;
  int prop_G;
  double prop_eps;
};

struct Params
{
  rgd::Box box;
  rgd::Grid grid;  // shape and inverse cell of the grids; data per atom in Comp::vdw_grid
  const double* ewald_grid;
  int quintic;  // the grids hold the 27 triquintic values per point (RG_SCHEME_TRIQUINTIC) instead of 8
  double overlap;
  float overlap_f;
  int use_charge;
  float hf[3][3];
  float rc2_mm, rc2_c, alpha, coul;
  int n_comp;
  Comp comp[kMaxComp];
  double beta, volume;
  double max_translation, max_rotation;
  double p_translation, p_rotation, p_swap, p_identity;
  int k1, k2, capacity, na;
  int nk;
  const char4* kvec;
  const double* temp;
  double uc[3][3], uic[3][3];
  int rep[3];
  // framework atoms, for trial atoms whose type has no VDW grid (explicit pairs; n_fw = 0 when every type has one)
  int n_fw;
  float rc2_fw;
  int km[3];       // kmax per axis: the phasor tables hold exp(2 pi i j s) for j = 0..km[d]
  int tabK;        // table stride: max(km) + 1
  int group;                // CTAs of this system in the launch; the system's CTA index is blockIdx.x % group
  int kpc;                  // k-vectors per CTA (the stride of the per-CTA k arrays in dynamic shared memory)
  int nslice;               // molecule sites of a CTA's slice staged in shared memory per phase (any rest from L2)
  int nseg_max;             // segments of a CTA's k-range at most (runs of up to kSegLen k-vectors sharing kx and ky)
  int ncand_max;            // Ewald candidates of a phase at most (the orientation trials)
  int cand_atoms;           // atoms of one candidate at most (old and new molecule: 2 x atoms per molecule)
  int cells;                // 1: the pair loop walks the 27 cells around each trial atom (0: every site of the slice)
  int nc[3];                // cells per axis, each at least the pair cutoff wide
};

// The state of one system: its molecules, running energy, statistics and structure factors, its launch flags and
// its copies of the pair table and framework atoms. Everything else (Params) is shared by the systems of one launch.
struct State
{
  unsigned long long seed;
  const float4* ljf;  // [kMaxTypes^2]: 4 eps, sigma^2, shift, lj flag
  const float* qtype; // charge per type (the pseudo-atom charge)
  const int4* fwx;    // [n_fw] fixed point, .w = type
  const float* fwq;   // [n_fw] charges
  double4* pos;    // [capacity * na] Cartesian
  int4* fx;        // [capacity * na] fixed point, .w = type | molecule << 8
  int* comp_of;    // [capacity]
  int* list;       // [kMaxComp][capacity]
  int* slot;       // [capacity]
  int* n_state;    // n, count[kMaxComp]
  double* energy;
  long long* move_base;
  double* stats;   // attempted[5], accepted[5], sum_n[4], sum_energy, samples
  double2* sk;     // [nk]
  double* part;    // [2][kRow][group]: partial sums, column-major, two buffers alternating by phase
  unsigned long long* bar;  // [0] barrier arrivals in this launch (zeroed before each launch), [1] error flag
  int record;
  long long spin_limit;     // polls before a barrier wait gives up (kSpinLimit; shorter only in the wait test)
  int absent_cta;           // wait test: this CTA does not arrive at the first barrier of a launch (-1: none)
};

// This CTA's system state, copied from global memory at the start of the launch (every device function reads it).
__shared__ State gs;

enum : uint32_t
{
  kKindMove = 1,
  kKindFirst = 2,
  kKindOrient = 3,
  kKindNewOrient = 4,
  kKindOldOrient = 5
};
__host__ __device__ constexpr uint32_t slot(uint32_t kind, uint32_t index, uint32_t sub)
{
  return (kind << 28) | (index << 8) | sub;
}

struct Shared
{
  float4 tab[kMaxTypes * kMaxTypes];
  float qt[kMaxTypes];
  double3 ta[kMaxItems];  // trial atoms: Cartesian position
  int4 tf[kMaxItems];     // fixed point, .w = type
  int nta;
  double3 cpos[kMaxCand][kMaxCandAtoms];  // Ewald candidates: atoms and signed charges
  double cq[kMaxCand][kMaxCandAtoms];
  int cn[kMaxCand];
  int ncand;
  double fwE[kMaxItems];              // framework (grid) energy of the trial atoms this CTA owns
  double red[kThreads];
  unsigned ovl_bits[4];
  double tot[kMaxItems + kMaxCand];  // totals over the grid
  unsigned ovl[4];
  // move state
  int kind, c, c2, m, axis, accept, fail, n, count[kMaxComp], gen;
  int phases;  // phases run by this CTA: its parity selects the buffer of partial-sum rows
  int nseg;    // segments of this CTA's k-range
  // molecule-list state an accepted deletion / identity change rewrites, read before the phase's barrier (no CTA
  // writes it before every CTA has passed that barrier, so every CTA reads the same values and writes the same update)
  int preSlot, preLastC, preCl, preSl;
  double3 preLast[kMaxAtoms];
  double u[8];
  double energy, dU;
  double3 mol[kMaxAtoms];   // new molecule (selected)
  double W, W2;
  int selFirst, selOrient;
  double3 first;
  double logq[kMaxTrials];
  double stats[kStats];
  double3 rel[kMaxTrials][kMaxAtoms];  // insertion: orientation offsets from the starting bead, computed up front
  int wsum[kWarps];                    // the pair warps' sums in the binning's prefix scan
  int staged_ns;                       // sites of the system when the slice in shared memory was staged (-1: none)
  int binned;                          // 1: the cells describe the staged slice as it is
};

__device__ __forceinline__ double2 urand(const Params& p, long long move, uint32_t sl)
{
  return rgd::uniform2(gs.seed, 0, move, sl);
}

__device__ __forceinline__ uint32_t fixOf(double s)
{
  s -= floor(s);
  return static_cast<uint32_t>(static_cast<unsigned long long>(s * 4294967296.0));
}
__device__ __forceinline__ int4 toFixed(const Params& p, double3 r, int w)
{
  const rgd::Box& b = p.box;
  const double s0 = b.ic[0][0] * r.x + b.ic[1][0] * r.y + b.ic[2][0] * r.z;
  const double s1 = b.ic[0][1] * r.x + b.ic[1][1] * r.y + b.ic[2][1] * r.z;
  const double s2 = b.ic[0][2] * r.x + b.ic[1][2] * r.y + b.ic[2][2] * r.z;
  return make_int4(static_cast<int>(fixOf(s0)), static_cast<int>(fixOf(s1)), static_cast<int>(fixOf(s2)), w);
}

// uniform rotation from three uniforms (Shoemake's unit quaternion)
__device__ void rotationFromUniforms(double u1, double u2, double u3, double R[3][3])
{
  double s2, c2, s3, c3;
  sincospi(2.0 * u2, &s2, &c2);
  sincospi(2.0 * u3, &s3, &c3);
  const double a = sqrt(1.0 - u1), b = sqrt(u1);
  const double x = a * s2, y = a * c2, z = b * s3, w = b * c3;
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

__device__ __forceinline__ unsigned long long loadAcquire(const unsigned long long* a)
{
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long loadRelaxed(const unsigned long long* a)
{
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long addRelease(unsigned long long* a, unsigned long long x)
{
  unsigned long long old;
  asm volatile("atom.add.release.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(a), "l"(x) : "memory");
  return old;
}

// Grid barrier over all CTAs of the cooperative launch: a monotonic arrival counter (zeroed before each launch); the
// n-th barrier of the launch is passed once the counter reaches n x group (the system's CTAs). One release add per CTA, then acquire
// polls: no reset, no second round trip. Spin-waits are bounded: on timeout the error flag is raised and false
// returned, and every CTA leaves the kernel; a CTA waiting on a barrier that a failed CTA will never reach sees the
// flag (polled every 64 spins) and leaves too.
__device__ bool gridBarrier(const Params& p, Shared& sh)
{
  __syncthreads();
  if (threadIdx.x == 0)
  {
    const unsigned long long target = static_cast<unsigned long long>(sh.gen + 1) * p.group;
    // the wait test leaves one arrival out of the first barrier, so that every CTA's bounded wait runs out
    const bool absent = static_cast<int>(blockIdx.x) % p.group == gs.absent_cta && sh.gen == 0;
    unsigned long long v = absent ? loadAcquire(&gs.bar[0]) : addRelease(&gs.bar[0], 1ull) + 1ull;
    long long spins = 0;
    while (v < target)
    {
      if (++spins > gs.spin_limit)
      {
        atomicExch(&gs.bar[1], 1ull);
        sh.fail = 1;
        break;
      }
      if ((spins & 63) == 0 && loadRelaxed(&gs.bar[1]) != 0ull)
      {
        sh.fail = 1;
        break;
      }
      __nanosleep(32);
      v = loadAcquire(&gs.bar[0]);
    }
    sh.gen += 1;
  }
  __syncthreads();
  return !sh.fail;
}

// Dynamic shared memory: the Ewald phasor tables (ncand_max x cand_atoms x 3 axes x tabK), this CTA's molecule
// sites staged per phase, its framework atoms (explicit pairs of grid-less types) kept for the launch, and its k-range.
struct Dyn
{
  double2* phasor;
  int4* slice;  // [nslice]
  int4* fws;    // [kFwSlice]
  float* fwq;   // [kFwSlice]
  double* eacc;  // [ncand_max][kThreads]: per thread its sum of each candidate's energy terms
  // this CTA's k-range for the whole launch: S(k) (only this CTA updates it; written back at the end of the launch),
  // the prefactors and the k-vectors
  double2* ks;  // [kpc]
  double* kt;   // [kpc]
  char4* kv;    // [kpc]
  int* segStart;  // [nseg_max + 1]: where each segment of the k-range starts, and (last) the range's length
  // the staged slice binned into cells, rebuilt every phase: where each cell's run starts in `order` (and, last, the
  // slice's length), per cell and pair warp the sites of the warp's part of the slice in that cell and then the
  // warp's write cursor there, and the slice indices in (cell, index) order
  int* cellStart;          // [ncell + 1]
  int* cellWarp;           // [ncell][kPairWarps]
  unsigned short* order;   // [nslice]
};
__host__ __device__ constexpr size_t phasorBytes(int tabK, int ncand, int catoms)
{
  return sizeof(double2) * static_cast<size_t>(ncand) * catoms * 3 * static_cast<size_t>(tabK);
}
__host__ __device__ constexpr size_t kRangeBytes(int kpc)
{
  return static_cast<size_t>(kpc) * (sizeof(double2) + sizeof(double) + sizeof(char4));
}
__host__ __device__ constexpr size_t cellBytes(int ncell, int nslice)
{
  return ncell == 0 ? 0
                    : sizeof(int) * ((kPairWarps + 1) * static_cast<size_t>(ncell) + 2) +
                          ((sizeof(unsigned short) * static_cast<size_t>(nslice) + 15) & ~size_t(15));
}
__host__ __device__ constexpr size_t dynBytes(int tabK, int ncand, int catoms, int kpc, int nseg, int nslice, int ncell)
{
  return phasorBytes(tabK, ncand, catoms) + sizeof(int4) * (static_cast<size_t>(nslice) + kFwSlice) +
         sizeof(float) * kFwSlice + sizeof(double) * static_cast<size_t>(ncand) * kThreads + kRangeBytes(kpc) +
         sizeof(int) * (static_cast<size_t>(nseg) + 2) + cellBytes(ncell, nslice);
}
__device__ __forceinline__ Dyn dynOf(const Params& p)
{
  extern __shared__ __align__(16) unsigned char dynSmem[];
  Dyn d;
  d.phasor = reinterpret_cast<double2*>(dynSmem);
  d.slice = reinterpret_cast<int4*>(dynSmem + phasorBytes(p.tabK, p.ncand_max, p.cand_atoms));
  d.fws = d.slice + p.nslice;
  d.fwq = reinterpret_cast<float*>(d.fws + kFwSlice);
  d.eacc = reinterpret_cast<double*>(d.fwq + kFwSlice);
  d.ks = reinterpret_cast<double2*>(d.eacc + p.ncand_max * kThreads);
  d.kt = reinterpret_cast<double*>(d.ks + p.kpc);
  d.kv = reinterpret_cast<char4*>(d.kt + p.kpc);
  const int ncell = p.cells ? p.nc[0] * p.nc[1] * p.nc[2] : 0;
  d.segStart = reinterpret_cast<int*>(d.kv + p.kpc);
  d.cellStart = d.segStart + p.nseg_max + 2;
  d.cellWarp = d.cellStart + (p.cells ? ncell + 2 : 0);
  d.order = reinterpret_cast<unsigned short*>(d.cellWarp + kPairWarps * ncell);
  return d;
}

// Structure-factor change of Ewald candidate c at the n <= kSegLen k-vectors kv[k0 ..] of one segment (they share kx
// and ky): per k the sum over the candidate's atoms of q exp(2 pi i k.s) (ewald.cpp:1043-1244), from the phasor tables
// of the current phase. Per atom the x and y phasors and the charge are multiplied once for the segment, then each k
// takes its z phasor; the kSegLen sums are independent. Entries u >= n repeat the last k-vector and are not used.
__device__ __forceinline__ void segmentDelta(const Params& p, const Shared& sh, const double2* phasor, const char4* kv,
                                             int c, int k0, int n, double2 (&d)[kSegLen])
{
  const char4 kb = kv[k0];
  int iz[kSegLen];
  bool neg[kSegLen];
#pragma unroll
  for (int u = 0; u < kSegLen; ++u)
  {
    const char4 k = kv[k0 + min(u, n - 1)];
    iz[u] = 2 * p.tabK + abs(k.z);
    neg[u] = k.z < 0;
    d[u] = make_double2(0.0, 0.0);
  }
  const int ix = abs(kb.x), iy = p.tabK + abs(kb.y);
  for (int a = 0; a < sh.cn[c]; ++a)
  {
    const double2* t = phasor + static_cast<long long>(c * p.cand_atoms + a) * 3 * p.tabK;
    double2 ex = t[ix], ey = t[iy];
    if (kb.x < 0) ex.y = -ex.y;
    if (kb.y < 0) ey.y = -ey.y;
    const double q = sh.cq[c][a];
    const double2 w = make_double2(q * (ex.x * ey.x - ex.y * ey.y), q * (ex.x * ey.y + ex.y * ey.x));
#pragma unroll
    for (int u = 0; u < kSegLen; ++u)
    {
      double2 z = t[iz[u]];
      if (neg[u]) z.y = -z.y;
      d[u].x += w.x * z.x - w.y * z.y;
      d[u].y += w.x * z.y + w.y * z.x;
    }
  }
}

// The accepted candidate's structure-factor change added to this CTA's S(k) range (the phasor tables of the phase
// that evaluated it are still in shared memory).
__device__ void addCandidate(const Params& p, const Shared& sh, const Dyn& dy, int c)
{
  for (int sg = threadIdx.x; sg < sh.nseg; sg += kThreads)
  {
    const int k0 = dy.segStart[sg], n = dy.segStart[sg + 1] - k0;
    double2 d[kSegLen];
    segmentDelta(p, sh, dy.phasor, dy.kv, c, k0, n, d);
#pragma unroll
    for (int u = 0; u < kSegLen; ++u)
      if (u < n)
      {
        dy.ks[k0 + u].x += d[u].x;
        dy.ks[k0 + u].y += d[u].y;
      }
  }
}

// Cell of a fixed-point fractional coordinate (uint32 x 2^-32) among nc cells along that axis, and the periodic wrap
// of a neighbouring cell index.
__device__ __forceinline__ int cellCoord(int f, int nc)
{
  return static_cast<int>((static_cast<unsigned long long>(static_cast<uint32_t>(f)) * static_cast<unsigned>(nc)) >> 32);
}
__device__ __forceinline__ int wrapCell(int c, int nc) { return c < 0 ? c + nc : (c >= nc ? c - nc : c); }
__device__ __forceinline__ int siteCell(const Params& p, int4 P)
{
  return cellCoord(P.x, p.nc[0]) + p.nc[0] * (cellCoord(P.y, p.nc[1]) + p.nc[1] * cellCoord(P.z, p.nc[2]));
}

// Squared distance of trial atom B and partner P (fixed point) in FP32 from the exact fixed-point displacement (the
// uint32 wrap is the minimum image).
// The launch constants the pair terms read, copied into registers once per phase by the pair warps (read through the
// Params reference they would be loaded again for every pair)
struct PairConst
{
  float hf[3][3];
  float overlap_f, rc2_c, alpha, coul;
  bool use_charge;
};
__device__ __forceinline__ PairConst pairConst(const Params& p)
{
  PairConst c;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) c.hf[a][b] = p.hf[a][b];
  c.overlap_f = p.overlap_f;
  c.rc2_c = p.rc2_c;
  c.alpha = p.alpha;
  c.coul = p.coul;
  c.use_charge = p.use_charge;
  return c;
}

template <class PC>
__device__ __forceinline__ float pairDistance2(const PC& p, int4 B, int4 P)
{
  const float f0 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.x) - static_cast<uint32_t>(P.x))) * kFix;
  const float f1 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.y) - static_cast<uint32_t>(P.y))) * kFix;
  const float f2 = static_cast<float>(static_cast<int>(static_cast<uint32_t>(B.z) - static_cast<uint32_t>(P.z))) * kFix;
  const float rx = fmaf(p.hf[0][0], f0, fmaf(p.hf[1][0], f1, p.hf[2][0] * f2));
  const float ry = fmaf(p.hf[0][1], f0, fmaf(p.hf[1][1], f1, p.hf[2][1] * f2));
  const float rz = fmaf(p.hf[0][2], f0, fmaf(p.hf[1][2], f1, p.hf[2][2] * f2));
  return fmaf(rx, rx, fmaf(ry, ry, rz * rz));
}

// Lennard-Jones + real-space Ewald of trial atom B (type bt, charge qb) with partner P at squared distance rr
// (.w & 0xff = type; charge qP), FP32, added to acc in FP64.
template <class PC>
__device__ __forceinline__ void pairEnergy(const PC& p, const Shared& sh, int bt, float qb, int4 P, float qP,
                                           float rr, float rc2v, double& acc, bool& ov)
{
  const int pt = P.w & 0xff;
  if (rr < rc2v)
  {
    const float4 q = sh.tab[bt * kMaxTypes + pt];
    if (q.w != 0.0f)
    {
      const float t = q.y * rgd::rcpRn(rr);
      const float t3 = t * t * t;
      const float e = q.x * (t3 * (t3 - 1.0f)) - q.z;
      if (e > p.overlap_f) ov = true;
      acc += static_cast<double>(e);
    }
  }
  if (p.use_charge && rr < p.rc2_c)
  {
    const float qq = qb * qP;
    if (qq != 0.0f)
    {
      // potentialCoulomb<0>, Ewald branch at full scaling: C qA qB erfc(alpha r) / r
      const float invr = rgd::rsqrtRn(rr);
      const float r = rr * invr;
      const float ex = expf(-p.alpha * p.alpha * rr);
      acc += static_cast<double>(p.coul * qq * rgd::erfcFromExp(p.alpha * r, ex) * invr);
    }
  }
}

template <class PC>
__device__ __forceinline__ void pairTerm(const PC& p, const Shared& sh, int4 B, int bt, float qb, int4 P, float qP,
                                         float rc2v, double& acc, bool& ov)
{
  pairEnergy(p, sh, bt, qb, P, qP, pairDistance2(p, B, P), rc2v, acc, ov);
}

// One phase: energies of sh.nta trial atoms (framework + molecules other than `skip`) and the Ewald energy change of
// sh.ncand candidates, each summed over the whole grid into sh.tot[0, nta) and sh.tot[nta, nta + ncand); overlap bits
// per trial atom in sh.ovl. vdwOf/qOf: the framework grid and charge of each trial atom (set by the caller in
// sh.tf[].w = type; the grids come from the type). Returns false if a barrier failed.
template <bool QUINTIC>  // the system's grids: triquintic (27 values per point) or tricubic (8)
__device__ bool phase(const Params& p, Shared& sh, int skip, const double* const* atomGrid)
{
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = p.group, cta = static_cast<int>(blockIdx.x) % p.group;
  const int nta = sh.nta, ncand = sh.ncand;
  const int ns = sh.n * p.na;
  const int chunk = (ns + G - 1) / G, s0 = min(ns, cta * chunk), s1 = min(ns, s0 + chunk);
  const int nst = min(s1 - s0, p.nslice);
  const Dyn dy = dynOf(p);
  if (tid < 4)
  {
    sh.ovl_bits[tid] = 0u;
    sh.ovl[tid] = 0u;
  }
  if (tid < nta) sh.fwE[tid] = 0.0;
  __syncthreads();
  // 0. framework grids of the trial atoms this CTA owns (b = cta, cta + G, ..), by 16 lanes of the last warp: lane l
  //    takes corner l & 7 of the VDW grid (l < 8) or of the unit-charge Ewald grid (l >= 8). Meanwhile the other warps
  //    stage this CTA's slice of molecule sites in shared memory and run the pairs (1.), so that the grid loads'
  //    latency overlaps them. The grid branch of interactions_framework_molecule.cpp: only an atom whose type has a
  //    VDW grid takes it (its charge term then comes from the Ewald grid); any other atom sees the framework atoms
  //    explicitly (below).
  double acc = 0.0;
  bool ov = false;
  int b = 0;
  if (warp == kWarps - 1)
  {
    // four trial atoms at a time, two per half-warp, so that their grid loads are in flight together
    const int half = lane >> 4, l16 = lane & 15;
    auto corner = [&](int b, double& q) -> double {
      const double* vdw = atomGrid[b];
      q = static_cast<double>(sh.qt[sh.tf[b].w & 0xff]);
      const bool charged = p.use_charge && p.ewald_grid != nullptr && q != 0.0;
      double v = 0.0;
      if (vdw != nullptr && (l16 < 8 || charged))
      {
        rgd::Grid g = p.grid;
        g.data = l16 < 8 ? vdw : p.ewald_grid;
        const double3 r = sh.ta[b];
        if (!QUINTIC)
          v = rgd::interpolateCorner(g, rgd::gridCell(g, r.x, r.y, r.z), l16 & 7);
        else if ((l16 & 7) == 0)  // triquintic grids: lanes 0 and 8 of the half take the whole interpolant
          v = rgd::interpolateQuintic(g, r.x, r.y, r.z, nullptr);
      }
      return v;
    };
    for (int b0 = cta; b0 < nta; b0 += 4 * G)
    {
      const int ba = b0 + half * G, bb = b0 + (2 + half) * G;
      double qa = 0.0, qbb = 0.0;
      double va = ba < nta ? corner(ba, qa) : 0.0;
      double vb = bb < nta ? corner(bb, qbb) : 0.0;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1)
      {
        va += __shfl_xor_sync(0xffffffffu, va, o);
        vb += __shfl_xor_sync(0xffffffffu, vb, o);
      }
      const double ewa = __shfl_sync(0xffffffffu, va, (lane & 16) | 8);
      const double ewb = __shfl_sync(0xffffffffu, vb, (lane & 16) | 8);
      if (l16 == 0 && ba < nta)
      {
        sh.fwE[ba] = va + qa * ewa;
        if (va > p.overlap) atomicOr(&sh.ovl_bits[ba >> 5], 1u << (ba & 31));
      }
      if (l16 == 0 && bb < nta)
      {
        sh.fwE[bb] = vb + qbb * ewb;
        if (vb > p.overlap) atomicOr(&sh.ovl_bits[bb >> 5], 1u << (bb & 31));
      }
    }
  }
  else
  {
    constexpr int kPairThreads = (kWarps - 1) * 32;
    // the slice stays in shared memory from phase to phase while the number of sites is unchanged (accepted moves
    // update it in place), and so do its cells while no site of it moved
    const bool fresh = sh.staged_ns == ns, binned = fresh && sh.binned;
    if (!fresh)
      for (int i = tid; i < nst; i += kPairThreads) dy.slice[i] = __ldcg(gs.fx + s0 + i);
    asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");  // the slice is staged (warps 0 .. kWarps - 2)
    if (tid == 0) sh.staged_ns = ns;
    // 1. molecule-molecule pairs over this CTA's slice of sites (staged part from shared memory, any rest from L2)
    const int streams = nta > 0 ? kPairThreads / nta : 0;
    b = nta > 0 ? tid % nta : 0;
    const int st = nta > 0 ? tid / nta : 0;
    const int n = s1 - s0;
    // cells pay off when the slice holds at least about two sites per cell
    const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
    const bool useCells = p.cells && n <= p.nslice && n >= 2 * ncell;
    if (useCells && !binned)
    {
      // the staged slice binned into cells at least the cutoff wide, as a stable counting sort: pair warp w takes the
      // w-th contiguous part of the slice and counts its sites per cell; a prefix scan over (cell, warp) in that order
      // (each pair thread scans a run of cells) gives every warp its cursor in every cell; then each warp scatters its
      // part in index order, so each cell lists its sites in slice order and the sums below are reproducible
      const int part = (n + kPairWarps - 1) / kPairWarps, i0 = min(n, warp * part), i1 = min(n, i0 + part);
      for (int c = tid; c < ncell * kPairWarps; c += kPairThreads) dy.cellWarp[c] = 0;
      asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");
      for (int i = i0 + lane; i < i1; i += 32) atomicAdd(&dy.cellWarp[siteCell(p, dy.slice[i]) * kPairWarps + warp], 1);
      asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");
      const int per = (ncell + kPairThreads - 1) / kPairThreads, c0 = min(ncell, tid * per), c1 = min(ncell, c0 + per);
      int run = 0;
      for (int c = c0 * kPairWarps; c < c1 * kPairWarps; ++c) run += dy.cellWarp[c];
      int incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1)
      {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) sh.wsum[warp] = incl;
      asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");
      int at = incl - run;
      for (int w = 0; w < warp; ++w) at += sh.wsum[w];
      for (int c = c0; c < c1; ++c)
      {
        dy.cellStart[c] = at;
        for (int w = 0; w < kPairWarps; ++w)
        {
          const int cnt = dy.cellWarp[c * kPairWarps + w];
          dy.cellWarp[c * kPairWarps + w] = at;
          at += cnt;
        }
      }
      if (tid == 0) dy.cellStart[ncell] = n;
      asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");
      for (int j0 = i0; j0 < i1; j0 += 32)
      {
        const int i = j0 + lane;
        const bool act = i < i1;
        const int c = act ? siteCell(p, dy.slice[i]) : -1 - lane;
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int base = act ? dy.cellWarp[c * kPairWarps + warp] : 0;
        __syncwarp();
        if (act)
        {
          dy.order[base + __popc(peers & ((1u << lane) - 1u))] = static_cast<unsigned short>(i);
          if (lane == 31 - __clz(peers)) dy.cellWarp[c * kPairWarps + warp] = base + __popc(peers);
        }
        __syncwarp();
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kPairThreads) : "memory");
      if (tid == 0) sh.binned = 1;
    }
    if (nta > 0 && st < streams)
    {
      const int4 B = sh.tf[b];
      const int bt = B.w & 0xff;
      const float qb = sh.qt[bt];
      const int ns_staged = min(n, p.nslice);
      const float rcut2 = p.use_charge ? fmaxf(p.rc2_mm, p.rc2_c) : p.rc2_mm;
      const float rc2mm = p.rc2_mm;
      const PairConst pc = pairConst(p);
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      if (useCells)
      {
        // the 27 cells around the trial atom (distinct: at least 3 cells per axis) shared among the atom's streams: with
        // fewer than 27 streams each walks every streams-th cell whole, with more each cell is split among
        // streams / 27 of them
        const int cstep = min(streams, 27), nsub = max(1, streams / 27);
        if (st < cstep * nsub)
        {
          const int cx = cellCoord(B.x, p.nc[0]), cy = cellCoord(B.y, p.nc[1]), cz = cellCoord(B.z, p.nc[2]);
          for (int k = st % cstep; k < 27; k += cstep)
          {
            const int c = wrapCell(cx + k % 3 - 1, p.nc[0]) +
                          p.nc[0] * (wrapCell(cy + (k / 3) % 3 - 1, p.nc[1]) + p.nc[1] * wrapCell(cz + k / 9 - 1, p.nc[2]));
            const int e = dy.cellStart[c + 1];
            int j = dy.cellStart[c] + st / cstep;
            // four sites of the cell per iteration: their distances without branches, then the energies of the few
            // within a cutoff, into four independent sums
            for (; j + 3 * nsub < e; j += 4 * nsub)
            {
              const int4 P0 = dy.slice[dy.order[j]], P1 = dy.slice[dy.order[j + nsub]],
                         P2 = dy.slice[dy.order[j + 2 * nsub]], P3 = dy.slice[dy.order[j + 3 * nsub]];
              const float r0 = (P0.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P0);
              const float r1 = (P1.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P1);
              const float r2 = (P2.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P2);
              const float r3 = (P3.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P3);
              if (fminf(fminf(r0, r1), fminf(r2, r3)) < rcut2)
              {
                if (r0 < rcut2) pairEnergy(pc, sh, bt, qb, P0, sh.qt[P0.w & 0xff], r0, rc2mm, a0, ov);
                if (r1 < rcut2) pairEnergy(pc, sh, bt, qb, P1, sh.qt[P1.w & 0xff], r1, rc2mm, a1, ov);
                if (r2 < rcut2) pairEnergy(pc, sh, bt, qb, P2, sh.qt[P2.w & 0xff], r2, rc2mm, a2, ov);
                if (r3 < rcut2) pairEnergy(pc, sh, bt, qb, P3, sh.qt[P3.w & 0xff], r3, rc2mm, a3, ov);
              }
            }
            for (; j < e; j += nsub)
            {
              const int4 P = dy.slice[dy.order[j]];
              if ((P.w >> 8) != skip) pairTerm(pc, sh, B, bt, qb, P, sh.qt[P.w & 0xff], rc2mm, a0, ov);
            }
          }
        }
      }
      else
      {
        int i = st;
        // staged sites, four per iteration: their distances without branches (the skipped molecule's at infinity),
        // then the energies of the few within a cutoff
        for (; i + 3 * streams < ns_staged; i += 4 * streams)
        {
          const int4 P0 = dy.slice[i], P1 = dy.slice[i + streams], P2 = dy.slice[i + 2 * streams],
                     P3 = dy.slice[i + 3 * streams];
          const float r0 = (P0.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P0);
          const float r1 = (P1.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P1);
          const float r2 = (P2.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P2);
          const float r3 = (P3.w >> 8) == skip ? INFINITY : pairDistance2(pc, B, P3);
          if (fminf(fminf(r0, r1), fminf(r2, r3)) < rcut2)
          {
            if (r0 < rcut2) pairEnergy(pc, sh, bt, qb, P0, sh.qt[P0.w & 0xff], r0, rc2mm, a0, ov);
            if (r1 < rcut2) pairEnergy(pc, sh, bt, qb, P1, sh.qt[P1.w & 0xff], r1, rc2mm, a1, ov);
            if (r2 < rcut2) pairEnergy(pc, sh, bt, qb, P2, sh.qt[P2.w & 0xff], r2, rc2mm, a2, ov);
            if (r3 < rcut2) pairEnergy(pc, sh, bt, qb, P3, sh.qt[P3.w & 0xff], r3, rc2mm, a3, ov);
          }
        }
        // the rest: remaining staged sites, then any beyond the staged slice from L2
        for (; i < n; i += streams)
        {
          const int4 P = i < p.nslice ? dy.slice[i] : __ldcg(gs.fx + s0 + i);
          if ((P.w >> 8) != skip) pairTerm(pc, sh, B, bt, qb, P, sh.qt[P.w & 0xff], rc2mm, a0, ov);
        }
      }
      acc = (a0 + a1) + (a2 + a3);
      // trial atom without a VDW grid: explicit pairs with this CTA's slice of the framework atoms
      if (p.n_fw > 0 && atomGrid[b] == nullptr)
      {
        const int fchunk = (p.n_fw + G - 1) / G, fa = min(p.n_fw, cta * fchunk), fb = min(p.n_fw, fa + fchunk);
        for (int j = st; j < fb - fa; j += streams)
        {
          const bool staged = j < kFwSlice;
          pairTerm(p, sh, B, bt, qb, staged ? dy.fws[j] : __ldg(gs.fwx + fa + j),
                   staged ? dy.fwq[j] : __ldg(gs.fwq + fa + j), p.rc2_fw, acc, ov);
        }
      }
    }
  }
  sh.red[tid] = acc;
  if (ov) atomicOr(&sh.ovl_bits[b >> 5], 1u << (b & 31));
  __syncthreads();
  // partial sums column-major ([column][CTA]), in two buffers alternating by phase: a CTA writes the next phase's
  // partials only after every CTA has passed this phase's barrier and read this phase's, which lie in the other buffer
  const int buf = sh.phases & 1;
  double* cols = gs.part + static_cast<long long>(buf) * kRow * G;
  if (tid < nta)
  {
    const int streams = (kWarps - 1) * 32 / nta;
    double s = 0.0;
    for (int k = 0; k < streams; ++k) s += sh.red[tid + nta * k];
    cols[static_cast<long long>(tid) * G + cta] = s + sh.fwE[tid];
  }
  if (tid < 4) cols[static_cast<long long>(kMaxItems + kMaxCand + tid) * G + cta] = static_cast<double>(sh.ovl_bits[tid]);
  // 2. Ewald candidates over this CTA's k-range. Per candidate atom (c, a) and axis d a phasor table
  //    tab[j] = exp(2 pi i j s_d), j = 0..kmax_d (j < 0: the conjugate), built by powers of tab[1] (one thread per
  //    table); then per (candidate, k) the structure-factor change sum_a q_a tab_x[kx] tab_y[ky] tab_z[kz] and its
  //    energy change (ewald.cpp:1043-1244), one thread each; then per candidate the sum over k in a fixed order.
  double2* phasor = dy.phasor;
  const int kchunk = (p.nk + G - 1) / G, k0 = cta * kchunk, nkr = max(0, min(p.nk, k0 + kchunk) - k0);
  if (ncand > 0)
  {
    const rgd::Box& bx = p.box;
    for (int task = tid; task < ncand * p.cand_atoms * 3; task += kThreads)
    {
      const int c = task / (p.cand_atoms * 3), a = (task / 3) % p.cand_atoms, d = task % 3;
      if (a >= sh.cn[c]) continue;
      const double3 r = sh.cpos[c][a];
      const double sd = bx.ic[0][d] * r.x + bx.ic[1][d] * r.y + bx.ic[2][d] * r.z;
      double sn, cs;
      sincospi(2.0 * sd, &sn, &cs);
      double2* t = phasor + (static_cast<long long>(c * p.cand_atoms + a) * 3 + d) * p.tabK;
      double2 w = make_double2(1.0, 0.0);
      t[0] = w;
      for (int j = 1; j <= p.km[d]; ++j)
      {
        w = make_double2(w.x * cs - w.y * sn, w.x * sn + w.y * cs);
        t[j] = w;
      }
    }
    __syncthreads();
    // energy change of each candidate over this CTA's k-range: one (candidate, segment) task at a time per thread,
    // its energy terms added to the thread's own sum for that candidate; then warp w sums candidates w and w + kWarps
    // over the threads in a fixed order
    const int nseg = sh.nseg;
    for (int c = 0; c < ncand; ++c) dy.eacc[c * kThreads + tid] = 0.0;
    for (int task = tid; task < ncand * nseg; task += kThreads)
    {
      const int c = task / nseg, sg = task - c * nseg;
      const int k0 = dy.segStart[sg], n = dy.segStart[sg + 1] - k0;
      double2 d[kSegLen];
      segmentDelta(p, sh, phasor, dy.kv, c, k0, n, d);
      double e = 0.0;
#pragma unroll
      for (int u = 0; u < kSegLen; ++u)
        if (u < n)
        {
          const double2 sk = dy.ks[k0 + u];
          e += dy.kt[k0 + u] * (2.0 * (sk.x * d[u].x + sk.y * d[u].y) + (d[u].x * d[u].x + d[u].y * d[u].y));
        }
      dy.eacc[c * kThreads + tid] += e;
    }
    __syncthreads();
    double esum0 = 0.0, esum1 = 0.0;
    if (warp < ncand)
      for (int j = lane; j < kThreads; j += 32) esum0 += dy.eacc[warp * kThreads + j];
    if (warp + kWarps < ncand)
      for (int j = lane; j < kThreads; j += 32) esum1 += dy.eacc[(warp + kWarps) * kThreads + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
      esum0 += __shfl_xor_sync(0xffffffffu, esum0, o);
      esum1 += __shfl_xor_sync(0xffffffffu, esum1, o);
    }
    if (lane == 0 && warp < ncand) cols[static_cast<long long>(kMaxItems + warp) * G + cta] = esum0;
    if (lane == 0 && warp + kWarps < ncand) cols[static_cast<long long>(kMaxItems + warp + kWarps) * G + cta] = esum1;
  }
  if (!gridBarrier(p, sh)) return false;
  // 3. totals: columns spread over the warps, lanes over the CTAs; all loads of a column are issued before any sum.
  //    The order is fixed (lane partials over j, then a fixed shuffle tree), so every CTA gets identical totals.
  const int nitems = nta + ncand, ncol = nitems + ((nta + 31) >> 5);
  constexpr int kU = 4;  // columns per warp with their loads in flight together
  for (int base = warp; base < ncol; base += kU * kWarps)
  {
    double v[kU][kMaxBlocks / 32];
#pragma unroll
    for (int u = 0; u < kU; ++u)
    {
      const int it = base + u * kWarps;
      const int col = min(kRow - 1, it < nta ? it : it < nitems ? kMaxItems + (it - nta) : kMaxItems + kMaxCand + (it - nitems));
      const double* src = cols + static_cast<long long>(col) * G;
#pragma unroll
      for (int j = 0; j < kMaxBlocks / 32; ++j)
      {
        const int q = lane + 32 * j;
        v[u][j] = (it < ncol && q < G) ? __ldcg(src + q) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < kU; ++u)
    {
      const int it = base + u * kWarps;
      if (it >= ncol) continue;
      if (it < nitems)
      {
        double sum = 0.0;
#pragma unroll
        for (int j = 0; j < kMaxBlocks / 32; ++j) sum += v[u][j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) sh.tot[it] = sum;
      }
      else
      {
        unsigned o = 0u;
#pragma unroll
        for (int j = 0; j < kMaxBlocks / 32; ++j) o |= static_cast<unsigned>(v[u][j]);
        o = __reduce_or_sync(0xffffffffu, o);
        if (lane == 0) sh.ovl[it - nitems] = o;
      }
    }
  }
  if (tid == 0) sh.phases += 1;
  __syncthreads();
  return true;
}

__device__ __forceinline__ bool ovlOf(const Shared& sh, int i) { return (sh.ovl[i >> 5] >> (i & 31)) & 1u; }

// Proposal density (relative to uniform) of a position for component c
__device__ double proposalDensity(const Params& p, const Comp& c, double3 r)
{
  const double v[3] = {r.x, r.y, r.z};
  int ci[3];
  for (int a = 0; a < 3; ++a)
  {
    const double s = rgd::fract1(p.uic[0][a] * v[0] + p.uic[1][a] * v[1] + p.uic[2][a] * v[2]);
    ci[a] = min(c.prop_G - 1, static_cast<int>(s * c.prop_G));
  }
  return c.prop_q[ci[0] + c.prop_G * (ci[1] + c.prop_G * ci[2])];
}

// First-bead trial position t of component c: uniform in the box, or from the component's tabulated proposal
__device__ double3 firstBeadPosition(const Params& p, const Comp& c, long long move, int t)
{
  const double2 a = urand(p, move, slot(kKindFirst, t, 0));
  const double2 b = urand(p, move, slot(kKindFirst, t, 1));
  const double2 u = urand(p, move, slot(kKindFirst, t, 2));
  double sf[3];
  const double(*cell)[3] = p.box.c;
  if (!c.prop_cdf || u.x < c.prop_eps)
  {
    sf[0] = a.x;
    sf[1] = a.y;
    sf[2] = b.x;
  }
  else
  {
    const double2 v = urand(p, move, slot(kKindFirst, t, 3));
    const int G = c.prop_G, ncell = G * G * G;
    int lo = 0, hi = ncell - 1;
    while (lo < hi)
    {
      const int mid = (lo + hi) >> 1;
      if (c.prop_cdf[mid] < u.y)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int ci = lo % G, cj = (lo / G) % G, ck = lo / (G * G);
    sf[0] = (ci + a.x) / G + static_cast<double>(min(p.rep[0] - 1, static_cast<int>(b.y * p.rep[0])));
    sf[1] = (cj + a.y) / G + static_cast<double>(min(p.rep[1] - 1, static_cast<int>(v.x * p.rep[1])));
    sf[2] = (ck + b.x) / G + static_cast<double>(min(p.rep[2] - 1, static_cast<int>(v.y * p.rep[2])));
    cell = p.uc;
  }
  return make_double3(cell[0][0] * sf[0] + cell[1][0] * sf[1] + cell[2][0] * sf[2],
                      cell[0][1] * sf[0] + cell[1][1] * sf[1] + cell[2][1] * sf[2],
                      cell[0][2] * sf[0] + cell[1][2] * sf[1] + cell[2][2] * sf[2]);
}

// orientation (kind, t) of component c as offsets from its starting bead: rel[i] = R o_i - R o_sb
__device__ void orientationOffsets(const Params& p, const Comp& c, long long move, uint32_t kind, int t, double3* rel)
{
  const double2 a = urand(p, move, slot(kind, t, 0));
  const double2 b = urand(p, move, slot(kind, t, 1));
  double R[3][3];
  rotationFromUniforms(a.x, a.y, b.x, R);
  const double* o0 = c.offsets[c.starting_bead];
  const double rc[3] = {R[0][0] * o0[0] + R[0][1] * o0[1] + R[0][2] * o0[2],
                        R[1][0] * o0[0] + R[1][1] * o0[1] + R[1][2] * o0[2],
                        R[2][0] * o0[0] + R[2][1] * o0[1] + R[2][2] * o0[2]};
  for (int i = 0; i < c.n_atoms; ++i)
  {
    const double* o = c.offsets[i];
    rel[i] = make_double3(R[0][0] * o[0] + R[0][1] * o[1] + R[0][2] * o[2] - rc[0],
                          R[1][0] * o[0] + R[1][1] * o[1] + R[1][2] * o[2] - rc[1],
                          R[2][0] * o[0] + R[2][1] * o[1] + R[2][2] * o[2] - rc[2]);
  }
}

// the atoms of component c with its starting bead at `first`, orientation from (kind, t)
__device__ void orientedMolecule(const Params& p, const Comp& c, double3 first, long long move, uint32_t kind, int t,
                                 double3* out)
{
  const double2 a = urand(p, move, slot(kind, t, 0));
  const double2 b = urand(p, move, slot(kind, t, 1));
  double R[3][3];
  rotationFromUniforms(a.x, a.y, b.x, R);
  const double* o0 = c.offsets[c.starting_bead];
  const double rc[3] = {R[0][0] * o0[0] + R[0][1] * o0[1] + R[0][2] * o0[2],
                        R[1][0] * o0[0] + R[1][1] * o0[1] + R[1][2] * o0[2],
                        R[2][0] * o0[0] + R[2][1] * o0[1] + R[2][2] * o0[2]};
  for (int i = 0; i < c.n_atoms; ++i)
  {
    const double* o = c.offsets[i];
    out[i] = make_double3(first.x - rc[0] + R[0][0] * o[0] + R[0][1] * o[1] + R[0][2] * o[2],
                          first.y - rc[1] + R[1][0] * o[0] + R[1][1] * o[1] + R[1][2] * o[2],
                          first.z - rc[2] + R[2][0] * o[0] + R[2][1] * o[1] + R[2][2] * o[2]);
  }
}

// Boltzmann selection among up to 32 trials held one per lane (CBMC::selectTrialPosition, cbmc/util.cpp:14-47): lane t
// holds the log-weight lw of trial t and whether it is allowed. Returns in every lane the selected trial (-1 if none)
// and W = sum over the allowed trials of exp(lw) / k. The maximum, the prefix sums and the total come from fixed
// shuffle patterns, so every CTA takes the same decision.
__device__ int warpSelect(double lw, bool ok, int k, double u, double* W)
{
  const int lane = threadIdx.x & 31;
  const bool on = ok && lane < k;
  double m = on ? lw : -1e300;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (m == -1e300)
  {
    *W = 0.0;
    return -1;
  }
  double pre = on ? exp(lw - m) : 0.0;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    const double y = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += y;
  }
  const double sum = __shfl_sync(0xffffffffu, pre, 31);
  *W = exp(m) * sum / static_cast<double>(k);
  const unsigned onMask = __ballot_sync(0xffffffffu, on);
  const unsigned hit = __ballot_sync(0xffffffffu, on && pre >= u * sum);
  return hit ? __ffs(hit) - 1 : 31 - __clz(onMask);
}

__device__ __forceinline__ double3 loadPos(const Params& p, int site)
{
  const double2* q = reinterpret_cast<const double2*>(gs.pos + site);
  const double2 a = __ldcg(q), b = __ldcg(q + 1);
  return make_double3(a.x, a.y, b.x);
}

// write the atoms of molecule m (every CTA writes the same values; each reads back only its own writes). Sites of
// this CTA's staged slice are updated in shared memory as well, which then needs new cells; a change of the number of
// molecules, made by the caller after this, moves every CTA's slice and so has it staged again.
__device__ void storeMolecule(const Params& p, Shared& sh, int m, int cidx, const double3* x)
{
  const Comp& c = p.comp[cidx];
  const int G = p.group, cta = static_cast<int>(blockIdx.x) % p.group;
  const int ns = sh.n * p.na, chunk = (ns + G - 1) / G, s0 = min(ns, cta * chunk), s1 = min(ns, s0 + chunk);
  const int nst = min(s1 - s0, p.nslice);
  int4* slice = dynOf(p).slice;
  for (int i = 0; i < p.na; ++i)
  {
    const int4 f = toFixed(p, x[i], c.types[i] | (m << 8));
    gs.pos[m * p.na + i] = make_double4(x[i].x, x[i].y, x[i].z, 0.0);
    gs.fx[m * p.na + i] = f;
    const int at = m * p.na + i - s0;
    if (sh.staged_ns == ns && at >= 0 && at < nst)
    {
      slice[at] = f;
      sh.binned = 0;
    }
  }
}

// the atoms of one orientation trial other than the starting bead, in atom order, into trial-atom slots base, base+1, ..
__device__ void storeOrientation(const Params& p, Shared& sh, const double** atomGrid, const Comp& cc,
                                 const double3* x, int base)
{
  int a = base;
  for (int i = 0; i < p.na; ++i)
  {
    if (i == cc.starting_bead) continue;
    sh.ta[a] = x[i];
    sh.tf[a] = toFixed(p, x[i], cc.types[i]);
    atomGrid[a] = cc.vdw_grid[i];
    ++a;
  }
}

// One launch: the parameters its systems share and each system's state (device copies); CTAs [s * group, (s + 1) *
// group) run system s.
constexpr int kMaxSystems = 148;  // independent systems of one launch (rg_mixture_run_many)
struct Launch
{
  Params p;
  const State* st[kMaxSystems];
};
static_assert(sizeof(Launch) <= 32000, "kernel parameter space");

template <bool QUINTIC>
__global__ void __launch_bounds__(kThreads, 1) mixtureKernel(const __grid_constant__ Launch L, int moves)
{
  const Params& p = L.p;
  const int cta = static_cast<int>(blockIdx.x) % p.group;
  if (threadIdx.x == 0) gs = *L.st[blockIdx.x / p.group];
  __syncthreads();
  __shared__ Shared sh;
  const int tid = threadIdx.x;
  const int na = p.na;
  for (int i = tid; i < kMaxTypes * kMaxTypes; i += kThreads) sh.tab[i] = gs.ljf[i];
  for (int i = tid; i < kMaxTypes; i += kThreads) sh.qt[i] = gs.qtype[i];
  if (tid == 0)
  {
    sh.n = gs.n_state[0];
    sh.staged_ns = -1;
    sh.binned = 0;
    for (int c = 0; c < kMaxComp; ++c) sh.count[c] = gs.n_state[1 + c];
    sh.energy = *gs.energy;
    sh.gen = 0;
    sh.fail = loadRelaxed(&gs.bar[1]) != 0ull;  // a barrier of an earlier launch timed out: do nothing
    sh.phases = 0;
    for (int k = 0; k < kStats; ++k) sh.stats[k] = gs.stats[k];
  }
  // this CTA's k-range
  const int G = p.group;
  const int kchunk = (p.nk + G - 1) / G, k0 = cta * kchunk, k1 = min(p.nk, k0 + kchunk);
  const long long move0 = *gs.move_base;
  __shared__ const double* atomGrid[kMaxItems];
  const Dyn dyk = dynOf(p);
  // this CTA's k-range and framework slice, kept in shared memory for the whole launch
  for (int kk = tid; kk < k1 - k0; kk += kThreads)
  {
    dyk.kv[kk] = p.kvec[k0 + kk];
    dyk.kt[kk] = p.temp[k0 + kk];
    dyk.ks[kk] = gs.sk[k0 + kk];
  }
  if (p.n_fw > 0)
  {
    const int fchunk = (p.n_fw + G - 1) / G, fa = min(p.n_fw, cta * fchunk);
    const int nf = min(min(p.n_fw, fa + fchunk) - fa, kFwSlice);
    const Dyn dy = dynOf(p);
    for (int i = tid; i < nf; i += kThreads)
    {
      dy.fws[i] = gs.fwx[fa + i];
      dy.fwq[i] = gs.fwq[fa + i];
    }
  }
  __syncthreads();
  // the k-range cut into segments: runs of k-vectors with the same kx and ky, each split into pieces of at most
  // kSegLen (the k-vectors are ordered by kx, ky, kz); the host sized nseg_max by the same rule
  if (tid == 0)
  {
    int ns = 0, runStart = 0;
    for (int kk = 0; kk < k1 - k0; ++kk)
    {
      const char4 a = dyk.kv[kk];
      const bool newRun = kk == 0 || a.x != dyk.kv[kk - 1].x || a.y != dyk.kv[kk - 1].y;
      if (newRun) runStart = kk;
      if (newRun || (kk - runStart) % kSegLen == 0)
      {
        if (ns < p.nseg_max) dyk.segStart[ns] = kk;
        ++ns;
      }
    }
    if (ns > p.nseg_max) sh.fail = 1;
    dyk.segStart[min(ns, p.nseg_max)] = max(0, k1 - k0);
    sh.nseg = min(ns, p.nseg_max);
  }
  __syncthreads();
  if (sh.fail) return;
  for (int mv = 0; mv < moves; ++mv)
  {
    const long long move = move0 + mv;
    // the move's eight uniform numbers: four Philox draws, one per lane of warp 0
    if (tid < 4)
    {
      const double2 u = urand(p, move, slot(kKindMove, 0, tid));
      sh.u[2 * tid] = u.x;
      sh.u[2 * tid + 1] = u.y;
    }
    if (tid < 32) __syncwarp();
    if (tid == 0)
    {
      sh.c = min(p.n_comp - 1, static_cast<int>(sh.u[0] * p.n_comp));
      const double ptot = p.p_translation + p.p_rotation + p.p_swap + p.p_identity;
      const double v = sh.u[1] * ptot;
      sh.kind = v < p.p_translation ? 0
                : v < p.p_translation + p.p_rotation ? 1
                : v < p.p_translation + p.p_rotation + p.p_swap ? (sh.u[2] < 0.5 ? 2 : 3)
                                                                 : 4;
      sh.accept = 0;
      sh.nta = 0;
      sh.ncand = 0;
    }
    __syncthreads();
    const int kind = sh.kind;
    int c = sh.c;
    if ((kind == 0 || kind == 1) && sh.count[c] > 0)
    {
      // translation (one Cartesian direction) or rotation (one Cartesian axis about the centre of mass)
      if (tid == 0)
      {
        const Comp& cc = p.comp[c];
        const int m = __ldcg(gs.list + c * p.capacity + min(sh.count[c] - 1, static_cast<int>(sh.u[3] * sh.count[c])));
        sh.m = m;
        const int dir = min(2, static_cast<int>(3.0 * sh.u[4]));
        double3 old[kMaxAtoms], nw[kMaxAtoms];
        for (int i = 0; i < na; ++i) old[i] = nw[i] = loadPos(p, m * na + i);
        if (kind == 0)
        {
          const double d = p.max_translation * 2.0 * (sh.u[5] - 0.5);
          for (int i = 0; i < na; ++i)
          {
            if (dir == 0) nw[i].x += d;
            if (dir == 1) nw[i].y += d;
            if (dir == 2) nw[i].z += d;
          }
        }
        else
        {
          const double ang = p.max_rotation * 2.0 * (sh.u[5] - 0.5);
          double sn, cs;
          sincos(ang, &sn, &cs);
          double ctr[3] = {0, 0, 0}, w = 0.0;
          for (int i = 0; i < na; ++i)
          {
            ctr[0] += cc.masses[i] * old[i].x;
            ctr[1] += cc.masses[i] * old[i].y;
            ctr[2] += cc.masses[i] * old[i].z;
            w += cc.masses[i];
          }
          for (int d = 0; d < 3; ++d) ctr[d] /= w;
          const int a1 = (dir + 1) % 3, a2 = (dir + 2) % 3;
          for (int i = 0; i < na; ++i)
          {
            const double dv[3] = {old[i].x - ctr[0], old[i].y - ctr[1], old[i].z - ctr[2]};
            double r[3] = {dv[0], dv[1], dv[2]};
            r[a1] = cs * dv[a1] - sn * dv[a2];
            r[a2] = sn * dv[a1] + cs * dv[a2];
            nw[i] = make_double3(ctr[0] + r[0], ctr[1] + r[1], ctr[2] + r[2]);
          }
        }
        for (int i = 0; i < na; ++i)
        {
          sh.ta[i] = nw[i];
          sh.tf[i] = toFixed(p, nw[i], cc.types[i]);
          atomGrid[i] = cc.vdw_grid[i];
          sh.ta[na + i] = old[i];
          sh.tf[na + i] = toFixed(p, old[i], cc.types[i]);
          atomGrid[na + i] = cc.vdw_grid[i];
          sh.cpos[0][i] = nw[i];
          sh.cq[0][i] = cc.charges[i];
          sh.cpos[0][na + i] = old[i];
          sh.cq[0][na + i] = -cc.charges[i];
          sh.mol[i] = nw[i];
        }
        sh.cn[0] = 2 * na;
        sh.nta = 2 * na;
        sh.ncand = p.use_charge ? 1 : 0;
      }
      __syncthreads();
      if (!phase<QUINTIC>(p, sh, sh.m, atomGrid)) break;
      if (tid == 0)
      {
        bool ovn = false;
        double dU = 0.0;
        for (int i = 0; i < na; ++i)
        {
          ovn |= ovlOf(sh, i);
          dU += sh.tot[i] - sh.tot[na + i];
        }
        if (p.use_charge) dU += sh.tot[sh.nta];
        if (!ovn && sh.u[6] < exp(-p.beta * dU))
        {
          sh.accept = 1;
          sh.energy += dU;
        }
      }
      __syncthreads();
      if (sh.accept)
      {
        if (tid == 0) storeMolecule(p, sh, sh.m, c, sh.mol);
        if (p.use_charge) addCandidate(p, sh, dyk, 0);
      }
    }
    else if (kind == 2 && sh.n < p.capacity)
    {
      // CBMC insertion: first-bead trials, then orientations about the selected bead
      const Comp& cc = p.comp[c];
      const int sb = cc.starting_bead;
      if (tid < p.k1)
      {
        const double3 r = firstBeadPosition(p, cc, move, tid);
        sh.ta[tid] = r;
        sh.tf[tid] = toFixed(p, r, cc.types[sb]);
        atomGrid[tid] = cc.vdw_grid[sb];
        sh.logq[tid] = cc.prop_cdf ? log(proposalDensity(p, cc, r)) : 0.0;
      }
      if (tid == 0)
      {
        sh.nta = p.k1;
        sh.ncand = 0;
      }
      // the orientations depend only on the move: their offsets are computed now, by threads of another warp
      if (tid >= 32 && tid < 32 + p.k2) orientationOffsets(p, cc, move, kKindOrient, tid - 32, sh.rel[tid - 32]);
      __syncthreads();
      if (!phase<QUINTIC>(p, sh, -1, atomGrid)) break;
      if (tid < 32)
      {
        const int t = tid;
        const double lw = t < p.k1 ? -p.beta * sh.tot[t] - sh.logq[t] : 0.0;
        double W;
        const int sel = warpSelect(lw, t < p.k1 && !ovlOf(sh, t), p.k1, urand(p, move, slot(kKindMove, 1, 0)).x, &W);
        if (tid == 0)
        {
          sh.selFirst = sel;
          sh.W = W;
        }
        if (tid == 0 && sel >= 0)
        {
          sh.first = sh.ta[sel];
          sh.dU = sh.tot[sel];
          sh.nta = p.k2 * (na - 1);
          sh.ncand = p.use_charge ? p.k2 : 0;
        }
      }
      __syncthreads();
      if (sh.selFirst >= 0)
      {
        // orientation trials, one per thread: the other atoms of each orientation; Ewald candidates: whole molecules
        if (tid < p.k2)
        {
          double3 x[kMaxAtoms];
          const double3 f = sh.first;
          for (int i = 0; i < na; ++i)
          {
            const double3 r = sh.rel[tid][i];
            x[i] = make_double3(f.x + r.x, f.y + r.y, f.z + r.z);
            sh.cpos[tid][i] = x[i];
            sh.cq[tid][i] = cc.charges[i];
          }
          sh.cn[tid] = na;
          storeOrientation(p, sh, atomGrid, cc, x, tid * (na - 1));
        }
        __syncthreads();
        if (!phase<QUINTIC>(p, sh, -1, atomGrid)) break;
        if (tid < 32)
        {
          const int per = na - 1, t = tid;
          double e = 0.0;
          bool o = false;
          if (t < p.k2)
            for (int i = 0; i < per; ++i)
            {
              e += sh.tot[t * per + i];
              o |= ovlOf(sh, t * per + i);
            }
          double W2;
          const int sel = warpSelect(-p.beta * e, t < p.k2 && !o, p.k2, urand(p, move, slot(kKindMove, 2, 0)).x, &W2);
          if (tid == 0 && sel >= 0 && sh.W * W2 >= 1e-150)
          {
            const double dEw = p.use_charge ? sh.tot[sh.nta + sel] + cc.self_excl : 0.0;
            const double W = sh.W * W2;
            const double pacc = exp(-p.beta * dEw) * p.beta * cc.fugacity * p.volume /
                                static_cast<double>(sh.count[c] + 1) * W / cc.w_ig;
            if (sh.u[6] < pacc)
            {
              double e = 0.0;
              for (int i = 0; i < per; ++i) e += sh.tot[sel * per + i];
              sh.accept = 1;
              sh.energy += sh.dU + e + dEw;
              sh.selOrient = sel;
              for (int i = 0; i < na; ++i) sh.mol[i] = sh.cpos[sel][i];
            }
          }
        }
        __syncthreads();
        if (sh.accept)
        {
          if (tid == 0)
          {
            const int m = sh.n;
            storeMolecule(p, sh, m, c, sh.mol);
            gs.comp_of[m] = c;
            gs.slot[m] = sh.count[c];
            gs.list[c * p.capacity + sh.count[c]] = m;
            sh.count[c] += 1;
            sh.n += 1;
          }
          if (p.use_charge) addCandidate(p, sh, dyk, sh.selOrient);
        }
      }
    }
    else if (kind == 3 && sh.count[c] > 0)
    {
      // CBMC deletion: first-bead retrace (trial 0 = old bead) and orientation retrace about the old bead
      const Comp& cc = p.comp[c];
      const int sb = cc.starting_bead;
      if (tid == 0) sh.m = __ldcg(gs.list + c * p.capacity + min(sh.count[c] - 1, static_cast<int>(sh.u[3] * sh.count[c])));
      __syncthreads();
      const int m = sh.m;
      if (tid < p.k1)
      {
        const double3 r = tid == 0 ? loadPos(p, m * na + sb) : firstBeadPosition(p, cc, move, tid);
        sh.ta[tid] = r;
        sh.tf[tid] = toFixed(p, r, cc.types[sb]);
        atomGrid[tid] = cc.vdw_grid[sb];
        sh.logq[tid] = cc.prop_cdf ? log(proposalDensity(p, cc, r)) : 0.0;
      }
      // list state and positions the update needs, read by threads of an idle warp in parallel
      {
        const int last = sh.n - 1, q = tid - 128;
        if (q == 0)
        {
          sh.preSlot = __ldcg(gs.slot + m);
          sh.cn[0] = na;
          sh.nta = p.k1 + p.k2 * (na - 1);
          sh.ncand = p.use_charge ? 1 : 0;
        }
        else if (q == 1)
          sh.preLastC = __ldcg(gs.list + c * p.capacity + sh.count[c] - 1);
        else if (q == 2)
          sh.preCl = __ldcg(gs.comp_of + last);
        else if (q == 3)
          sh.preSl = __ldcg(gs.slot + last);
        else if (q >= 4 && q < 4 + na)
          sh.preLast[q - 4] = loadPos(p, last * na + (q - 4));
        else if (q >= 8 && q < 8 + na)
        {
          sh.cpos[0][q - 8] = loadPos(p, m * na + (q - 8));
          sh.cq[0][q - 8] = -cc.charges[q - 8];
        }
      }
      // retrace orientations about the old first bead, one per thread (trial 0: the molecule itself)
      if (tid < p.k2)
      {
        double3 x[kMaxAtoms];
        if (tid == 0)
          for (int i = 0; i < na; ++i) x[i] = loadPos(p, m * na + i);
        else
          orientedMolecule(p, cc, loadPos(p, m * na + sb), move, kKindOrient, tid, x);
        storeOrientation(p, sh, atomGrid, cc, x, p.k1 + tid * (na - 1));
      }
      __syncthreads();
      if (!phase<QUINTIC>(p, sh, m, atomGrid)) break;
      if (tid < 32)
      {
        // Rosenbluth weights of the retrace: first beads (trial 0 = the old bead) and orientations (trial 0 = the
        // molecule itself); lane t holds trial t of each
        const int t = tid, per = na - 1;
        const bool ok1 = t < p.k1 && !ovlOf(sh, t);
        double W1, W2;
        warpSelect(t < p.k1 ? -p.beta * sh.tot[t] - sh.logq[t] : 0.0, ok1, p.k1, 0.0, &W1);
        double e = 0.0;
        bool o = false;
        if (t < p.k2)
          for (int i = 0; i < per; ++i)
          {
            e += sh.tot[p.k1 + t * per + i];
            o |= ovlOf(sh, p.k1 + t * per + i);
          }
        warpSelect(-p.beta * e, t < p.k2 && !o, p.k2, 0.0, &W2);
        const bool ok2 = !o;
        if (tid == 0 && ok1 && ok2)
        {
          const double e0 = e;
          const double dEw = p.use_charge ? sh.tot[sh.nta] - cc.self_excl : 0.0;
          const double W = W1 * W2;
          const double pacc = exp(-p.beta * dEw) * static_cast<double>(sh.count[c]) /
                              (p.beta * cc.fugacity * p.volume) * cc.w_ig / W;
          if (sh.u[6] < pacc)
          {
            sh.accept = 1;
            sh.energy += -(sh.tot[0] + e0) + dEw;
          }
        }
      }
      __syncthreads();
      if (sh.accept)
      {
        if (tid == 0)
        {
          // remove m from its component list, then move the last molecule into slot m (from the values read before
          // the barrier)
          const int k = sh.preSlot, lastC = sh.preLastC;
          gs.list[c * p.capacity + k] = lastC;
          gs.slot[lastC] = k;
          sh.count[c] -= 1;
          const int last = sh.n - 1;
          if (m != last)
          {
            const int cl = sh.preCl;
            const int sl = (lastC == last) ? k : sh.preSl;
            storeMolecule(p, sh, m, cl, sh.preLast);
            gs.comp_of[m] = cl;
            gs.slot[m] = sl;
            gs.list[cl * p.capacity + sl] = m;
          }
          sh.n -= 1;
        }
        if (p.use_charge) addCandidate(p, sh, dyk, 0);
      }
    }
    else if (kind == 4 && p.n_comp > 1)
    {
      // identity change: old and new component swapped with probability 1/2 (identity_change.cpp:62-66)
      if (tid == 0)
      {
        int oldC = c, newC = (c + 1 + min(p.n_comp - 2, static_cast<int>(sh.u[3] * (p.n_comp - 1)))) % p.n_comp;
        if (sh.u[4] < 0.5)
        {
          const int t = oldC;
          oldC = newC;
          newC = t;
        }
        sh.c = oldC;
        sh.c2 = newC;
        sh.m = sh.count[oldC] > 0
                   ? __ldcg(gs.list + oldC * p.capacity +
                            min(sh.count[oldC] - 1, static_cast<int>(sh.u[5] * sh.count[oldC])))
                   : -1;
      }
      __syncthreads();
      if (sh.m >= 0)
      {
        const int m = sh.m, oldC = sh.c, newC = sh.c2;
        const Comp& co = p.comp[oldC];
        const Comp& cn = p.comp[newC];
        // trial atoms: new first bead (on the old starting bead), new orientations, old first bead, old retrace; the
        // orientations are built one per thread (new: threads [0, k2), old: threads [k2, 2 k2))
        const int base2 = 1 + p.k2 * (na - 1);  // slot of the old first bead
        const double3 first = loadPos(p, m * na + co.starting_bead);
        if (tid == 0)
        {
          sh.preSlot = __ldcg(gs.slot + m);
          sh.preLastC = __ldcg(gs.list + oldC * p.capacity + sh.count[oldC] - 1);
          sh.ta[0] = first;
          sh.tf[0] = toFixed(p, first, cn.types[cn.starting_bead]);
          atomGrid[0] = cn.vdw_grid[cn.starting_bead];
          sh.ta[base2] = first;
          sh.tf[base2] = toFixed(p, first, co.types[co.starting_bead]);
          atomGrid[base2] = co.vdw_grid[co.starting_bead];
          sh.nta = 2 * base2;
          sh.ncand = p.use_charge ? p.k2 : 0;
        }
        if (tid < p.k2)
        {
          const int t = tid;
          double3 x[kMaxAtoms];
          orientedMolecule(p, cn, first, move, kKindNewOrient, t, x);
          for (int i = 0; i < na; ++i)
          {
            sh.cpos[t][i] = x[i];
            sh.cq[t][i] = cn.charges[i];
            sh.cpos[t][na + i] = loadPos(p, m * na + i);
            sh.cq[t][na + i] = -co.charges[i];
          }
          sh.cn[t] = 2 * na;
          storeOrientation(p, sh, atomGrid, cn, x, 1 + t * (na - 1));
        }
        else if (tid < 2 * p.k2)
        {
          const int t = tid - p.k2;
          double3 x[kMaxAtoms];
          if (t == 0)
            for (int i = 0; i < na; ++i) x[i] = loadPos(p, m * na + i);
          else
            orientedMolecule(p, co, first, move, kKindOldOrient, t, x);
          storeOrientation(p, sh, atomGrid, co, x, base2 + 1 + t * (na - 1));
        }
        __syncthreads();
        if (!phase<QUINTIC>(p, sh, m, atomGrid)) break;
        if (tid < 32)
        {
          const int per = na - 1;
          // lane t: new orientation t and old retrace orientation t (trial 0 = the molecule itself)
          const int t = tid;
          double e = 0.0, eo = 0.0;
          bool o = false, oo = false;
          if (t < p.k2)
            for (int i = 0; i < per; ++i)
            {
              e += sh.tot[1 + t * per + i];
              o |= ovlOf(sh, 1 + t * per + i);
              eo += sh.tot[base2 + 1 + t * per + i];
              oo |= ovlOf(sh, base2 + 1 + t * per + i);
            }
          double Wn2, Wo2;
          const int sel = warpSelect(-p.beta * e, t < p.k2 && !o, p.k2, urand(p, move, slot(kKindMove, 3, 0)).x, &Wn2);
          warpSelect(-p.beta * eo, t < p.k2 && !oo, p.k2, 0.0, &Wo2);
          const double eSel = __shfl_sync(0xffffffffu, e, sel >= 0 ? sel : 0);
          const double e0 = eo;  // lane 0: the old molecule's own orientation
          const bool newFirstOk = !ovlOf(sh, 0), oldOk = !ovlOf(sh, base2) && !oo;
          const double Wn = exp(-p.beta * sh.tot[0]) * Wn2, Wo = exp(-p.beta * sh.tot[base2]) * Wo2;
          if (tid == 0 && newFirstOk && sel >= 0 && oldOk && Wn >= 1e-150)
          {
            const double dEw = p.use_charge ? sh.tot[sh.nta + sel] + cn.self_excl - co.self_excl : 0.0;
            const double pacc = exp(-p.beta * dEw) * (Wn / cn.w_ig) * cn.fugacity *
                                static_cast<double>(sh.count[oldC]) /
                                ((Wo / co.w_ig) * co.fugacity * static_cast<double>(sh.count[newC] + 1));
            if (sh.u[6] < pacc)
            {
              const double en = sh.tot[0] + eSel;
              sh.accept = 1;
              sh.energy += (en - (sh.tot[base2] + e0)) + dEw;
              sh.selOrient = sel;
              for (int i = 0; i < na; ++i) sh.mol[i] = sh.cpos[sel][i];
            }
          }
        }
        __syncthreads();
        if (sh.accept)
        {
          if (tid == 0)
          {
            storeMolecule(p, sh, m, newC, sh.mol);
            // move m from the old component's list to the new one's (from the values read before the barrier)
            const int k = sh.preSlot, lastC = sh.preLastC;
            gs.list[oldC * p.capacity + k] = lastC;
            gs.slot[lastC] = k;
            sh.count[oldC] -= 1;
            gs.comp_of[m] = newC;
            gs.slot[m] = sh.count[newC];
            gs.list[newC * p.capacity + sh.count[newC]] = m;
            sh.count[newC] += 1;
          }
          if (p.use_charge) addCandidate(p, sh, dyk, sh.selOrient);
        }
        c = oldC;
      }
    }
    __syncthreads();
    if (tid == 0 && gs.record)
    {
      sh.stats[kind] += 1.0;
      sh.stats[5 + kind] += sh.accept ? 1.0 : 0.0;
      for (int q = 0; q < p.n_comp && q < 4; ++q) sh.stats[10 + q] += sh.count[q];
      sh.stats[14] += sh.energy;
      sh.stats[15] += 1.0;
    }
    __syncthreads();
  }
  for (int kk = tid; kk < k1 - k0; kk += kThreads) gs.sk[k0 + kk] = dyk.ks[kk];
  if (cta == 0 && tid == 0 && !sh.fail)
  {
    gs.n_state[0] = sh.n;
    for (int c = 0; c < kMaxComp; ++c) gs.n_state[1 + c] = sh.count[c];
    *gs.energy = sh.energy;
    *gs.move_base = move0 + moves;
    for (int k = 0; k < kStats; ++k) gs.stats[k] = sh.stats[k];
  }
}
}  // namespace

struct rg_mixture
{
  rg_ctx* ctx = nullptr;
  rg_system* system = nullptr;
  rg_ewald* ewald = nullptr;
  Params p{};
  State st{};
  State* d_st = nullptr;  // device copy of st, refreshed before each launch
  int blocks = 0;
  int n_comp = 0;
  size_t smem = 0;  // dynamic shared memory of a launch: the Ewald phasor tables
  std::vector<void*> allocs;
};

namespace
{
void freeAll(rg_mixture* x)
{
  for (void* q : x->allocs) cudaFree(q);
  x->allocs.clear();
}
}  // namespace

extern "C" rg_status rg_mixture_create(rg_system* system, rg_ewald* ewald, const rg_gcmc_component* comps,
                                       int n_components, const rg_mixture_params* params, const double* xyz,
                                       const int32_t* comp_of_molecule, int n_molecules, rg_mixture** out)
{
  if (!system || !comps || !params || !out || n_components < 1 || n_components > kMaxComp || n_molecules < 0 ||
      (n_molecules > 0 && (!xyz || !comp_of_molecule)))
    return RG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  rgd::FF ff{};
  rgd::Box box{};
  const double* tg[64] = {};
  const double* eg = nullptr;
  int nt = 0, gd[3] = {0, 0, 0};
  double gic[3][3];
  rg_ctx* ctx = nullptr;
  rg_status st = rgd::systemExport(system, &ff, &box, tg, &eg, &nt, gd, gic, &ctx);
  if (st) return st;
  if (nt > kMaxTypes) return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_mixture: at most 16 pseudo-atom types");
  const int na = comps[0].n_atoms;
  if (na < 2 || na > kMaxAtoms) return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_mixture: molecules of 2-4 atoms");
  for (int c = 0; c < n_components; ++c)
    if (comps[c].n_atoms != na || comps[c].starting_bead < 0 || comps[c].starting_bead >= na)
      return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_mixture: every component needs the same atom count");
  if (params->n_first_bead_trials < 1 || params->n_first_bead_trials > kMaxTrials ||
      params->n_orientation_trials < 1 || params->n_orientation_trials > kMaxTrials)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: 1..12 first-bead and orientation trials");
  if (2 + 2 * params->n_orientation_trials * (na - 1) > kMaxItems ||
      params->n_first_bead_trials + params->n_orientation_trials * (na - 1) > kMaxItems)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: too many trial atoms per phase");
  if (params->max_molecules < n_molecules || params->max_molecules < 1 || params->max_molecules > (1 << 22))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: max_molecules");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  auto* x = new rg_mixture();
  x->ctx = ctx;
  x->system = system;
  x->ewald = ewald;
  x->n_comp = n_components;
  Params& p = x->p;
  p.box = box;
  p.grid.nx = gd[0];
  p.grid.ny = gd[1];
  p.grid.nz = gd[2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      p.grid.ic[i][j] = gic[i][j];
      p.hf[i][j] = static_cast<float>(box.c[i][j]);
    }
  p.ewald_grid = eg;
  p.quintic = rgd::systemScheme(system) == RG_SCHEME_TRIQUINTIC ? 1 : 0;
  p.overlap = ff.overlap;
  p.overlap_f = static_cast<float>(ff.overlap);
  p.use_charge = (ff.use_charge && ewald) ? 1 : 0;
  p.beta = params->beta;
  p.volume = box.volume;
  p.max_translation = params->max_translation;
  p.max_rotation = params->max_rotation;
  p.p_translation = params->p_translation;
  p.p_rotation = params->p_rotation;
  p.p_swap = params->p_swap;
  p.p_identity = params->p_identity;
  p.k1 = params->n_first_bead_trials;
  p.k2 = params->n_orientation_trials;
  p.capacity = params->max_molecules;
  p.na = na;
  p.n_comp = n_components;
  x->st.seed = params->seed;
  // pair table (FP32) and the charge of each type
  std::vector<float4> ljf(kMaxTypes * kMaxTypes, make_float4(0, 0, 0, 0));
  std::vector<float> qtype(kMaxTypes, 0.0f);
  {
    std::vector<double> eps4(nt * nt), sig2(nt * nt), shift(nt * nt);
    std::vector<int> lj(nt * nt);
    cudaError_t e = cudaMemcpy(eps4.data(), ff.eps4, sizeof(double) * nt * nt, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(sig2.data(), ff.sig2, sizeof(double) * nt * nt, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(shift.data(), ff.shift, sizeof(double) * nt * nt, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lj.data(), ff.lj, sizeof(int) * nt * nt, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
    {
      delete x;
      return rg::cudaFail(ctx, e, "rg_mixture_create: pair table");
    }
    for (int a = 0; a < nt; ++a)
      for (int b = 0; b < nt; ++b)
        if (lj[a * nt + b])
          ljf[a * kMaxTypes + b] = make_float4(static_cast<float>(eps4[a * nt + b]), static_cast<float>(sig2[a * nt + b]),
                                               static_cast<float>(shift[a * nt + b]), 1.0f);
  }
  const double rcv_mol = params->cutoff_molecule_vdw, rcc = params->cutoff_coulomb;
  p.rc2_mm = static_cast<float>(rcv_mol * rcv_mol);
  p.rc2_c = static_cast<float>(rcc * rcc);
  p.rc2_fw = static_cast<float>(params->cutoff_framework_vdw * params->cutoff_framework_vdw);
  p.alpha = static_cast<float>(ff.alpha);
  p.coul = static_cast<float>(ff.coul);
  // components
  double ewaldAlpha = ff.alpha;
  for (int c = 0; c < n_components; ++c)
  {
    const rg_gcmc_component& q = comps[c];
    Comp& cc = p.comp[c];
    cc.n_atoms = q.n_atoms;
    cc.starting_bead = q.starting_bead;
    for (int i = 0; i < q.n_atoms; ++i)
    {
      cc.types[i] = q.types[i];
      cc.charges[i] = q.charges[i];
      cc.masses[i] = q.masses[i];
      for (int d = 0; d < 3; ++d) cc.offsets[i][d] = q.offsets[3 * i + d];
      cc.vdw_grid[i] = (q.types[i] >= 0 && q.types[i] < 64) ? tg[q.types[i]] : nullptr;
      if (q.types[i] < 0 || q.types[i] >= nt)
      {
        delete x;
        return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: component atom type");
      }
      qtype[q.types[i]] = static_cast<float>(q.charges[i]);
    }
    cc.fugacity = params->fugacity[c];
    cc.w_ig = params->w_ig[c] > 0.0 ? params->w_ig[c] : 1.0;
    // Ewald self + intramolecular exclusion energy of one molecule (ewald.cpp:1164-1238, new-atom terms)
    double self = 0.0, excl = 0.0;
    const double C = rg::coulombFactor();
    for (int i = 0; i < q.n_atoms; ++i) self -= C * ewaldAlpha * rg::kInvSqrtPi * q.charges[i] * q.charges[i];
    for (int i = 0; i < q.n_atoms; ++i)
      for (int j = i + 1; j < q.n_atoms; ++j)
      {
        double d2 = 0.0;
        for (int k = 0; k < 3; ++k)
        {
          const double d = q.offsets[3 * i + k] - q.offsets[3 * j + k];
          d2 += d * d;
        }
        const double r = std::sqrt(d2);
        excl -= C * q.charges[i] * q.charges[j] * std::erf(ewaldAlpha * r) / r;
      }
    cc.self_excl = self + excl;
  }
  // framework atoms in fixed point, needed only if some component atom type has no VDW grid
  bool gridless = false;
  for (int c = 0; c < n_components; ++c)
    for (int i = 0; i < na; ++i) gridless |= p.comp[c].vdw_grid[i] == nullptr;
  std::vector<int4> hfw;
  std::vector<float> hfq;
  {
    const rg_atom* dfw = nullptr;
    int nfw = 0;
    st = rgd::systemFramework(system, &dfw, &nfw);
    if (st)
    {
      delete x;
      return st;
    }
    if (gridless && nfw > 0)
    {
      std::vector<rg_atom> fw(nfw);
      const cudaError_t e = cudaMemcpy(fw.data(), dfw, sizeof(rg_atom) * nfw, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess)
      {
        delete x;
        return rg::cudaFail(ctx, e, "rg_mixture_create: framework atoms");
      }
      hfw.resize(nfw);
      hfq.resize(nfw);
      for (int i = 0; i < nfw; ++i)
      {
        if (fw[i].type >= nt)
        {
          delete x;
          return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: framework atom type");
        }
        const double r[3] = {fw[i].x, fw[i].y, fw[i].z};
        int f[3];
        for (int a = 0; a < 3; ++a)
        {
          const double sa = box.ic[0][a] * r[0] + box.ic[1][a] * r[1] + box.ic[2][a] * r[2];
          const double v = sa - std::floor(sa);
          f[a] = static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(v * 4294967296.0)));
        }
        hfw[i] = make_int4(f[0], f[1], f[2], fw[i].type);
        hfq[i] = static_cast<float>(fw[i].charge);
      }
    }
  }
  p.n_fw = static_cast<int>(hfw.size());
  // Ewald tables
  if (p.use_charge)
  {
    const char4* kv = nullptr;
    const double* temp = nullptr;
    const double2* srig = nullptr;
    int64_t nk = 0;
    int kmax[3];
    double alpha, sis;
    st = rgd::ewaldExport(ewald, &kv, &temp, &srig, &nk, kmax, &alpha, &sis);
    if (st)
    {
      delete x;
      return st;
    }
    p.kvec = kv;
    p.temp = temp;
    p.nk = static_cast<int>(nk);
    for (int d = 0; d < 3; ++d) p.km[d] = kmax[d];
  }
  p.tabK = 1 + std::max({p.km[0], p.km[1], p.km[2]});
  // launch geometry: one CTA per SM, co-resident; this system's CTAs split its k-vectors into ranges of kpc
  int sms = 0, perSM = 0;
  cudaError_t err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (err != cudaSuccess)
  {
    delete x;
    return rg::cudaFail(ctx, err, "rg_mixture_create");
  }
  x->blocks = std::min(kMaxBlocks, params->n_blocks > 0 ? std::min(params->n_blocks, sms) : sms);
  p.group = x->blocks;
  p.kpc = std::max(1, (p.nk + x->blocks - 1) / x->blocks);
  // segments of each CTA's k-range, cut by the kernel's rule (runs of equal kx and ky, pieces of at most kSegLen):
  // their largest count sizes the segment table in shared memory
  p.nseg_max = 0;
  if (p.use_charge && p.nk > 0)
  {
    std::vector<char4> hk(static_cast<size_t>(p.nk));
    err = cudaMemcpyAsync(hk.data(), p.kvec, sizeof(char4) * hk.size(), cudaMemcpyDeviceToHost, ctx->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
    if (err != cudaSuccess)
    {
      delete x;
      return rg::cudaFail(ctx, err, "rg_mixture_create");
    }
    for (int cta = 0; cta < x->blocks; ++cta)
    {
      const int k0 = cta * p.kpc, k1 = std::min(p.nk, k0 + p.kpc);
      int ns = 0, runStart = 0;
      for (int kk = 0; kk < k1 - k0; ++kk)
      {
        const char4 a = hk[k0 + kk];
        const bool newRun = kk == 0 || a.x != hk[k0 + kk - 1].x || a.y != hk[k0 + kk - 1].y;
        if (newRun) runStart = kk;
        if (newRun || (kk - runStart) % kSegLen == 0) ++ns;
      }
      p.nseg_max = std::max(p.nseg_max, ns);
    }
  }
  // shared memory: the k-range must fit; the staged slice of molecule sites takes what is left, up to a CTA's share of
  // a full system (sites beyond the slice are read from L2)
  cudaFuncAttributes fa{};
  int optin = 0;
  err = cudaFuncGetAttributes(&fa, p.quintic ? mixtureKernel<true> : mixtureKernel<false>);
  if (err == cudaSuccess) err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
  if (err != cudaSuccess)
  {
    delete x;
    return rg::cudaFail(ctx, err, "rg_mixture_create");
  }
  // cells of the pair loop: at least the largest pair cutoff wide along each perpendicular width, at most kMaxCells in
  // all (wider cells are still valid), and used only with at least 3 per axis (the 27 neighbours must be distinct)
  {
    const double rcut = std::sqrt(static_cast<double>(p.use_charge ? std::max(p.rc2_mm, p.rc2_c) : p.rc2_mm));
    double w[3];
    for (int a = 0; a < 3; ++a)
    {
      const int b1 = (a + 1) % 3, b2 = (a + 2) % 3;
      const double cr[3] = {box.c[b1][1] * box.c[b2][2] - box.c[b1][2] * box.c[b2][1],
                            box.c[b1][2] * box.c[b2][0] - box.c[b1][0] * box.c[b2][2],
                            box.c[b1][0] * box.c[b2][1] - box.c[b1][1] * box.c[b2][0]};
      w[a] = box.volume / std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      const double n = rcut > 0.0 ? std::floor(w[a] / rcut) : 0.0;
      p.nc[a] = static_cast<int>(std::min<double>(n, kMaxCells));
    }
    while (static_cast<long long>(p.nc[0]) * p.nc[1] * p.nc[2] > kMaxCells)
    {
      const int a = (p.nc[0] >= p.nc[1] && p.nc[0] >= p.nc[2]) ? 0 : (p.nc[1] >= p.nc[2] ? 1 : 2);
      p.nc[a] -= 1;
    }
    p.cells = (p.nc[0] >= 3 && p.nc[1] >= 3 && p.nc[2] >= 3) ? 1 : 0;
  }
  // the Ewald candidates of a phase: up to k2 orientations (insertion, identity change) or one molecule, each of at
  // most the old and the new molecule's atoms
  p.ncand_max = std::max(1, p.k2);
  p.cand_atoms = 2 * na;
  const long long budget = static_cast<long long>(optin) - static_cast<long long>(fa.sharedSizeBytes) - 1024;
  auto fixedOf = [&](int cells) {
    return static_cast<long long>(
               dynBytes(p.tabK, p.ncand_max, p.cand_atoms, p.kpc, p.nseg_max, 0, cells ? p.nc[0] * p.nc[1] * p.nc[2] : 0)) +
           16;
  };
  auto perSiteOf = [&](int cells) { return static_cast<long long>(sizeof(int4) + (cells ? sizeof(unsigned short) : 0)); };
  // without room for the cells next to the k-range, the pair loop walks the slice as it is
  if (p.cells && fixedOf(1) + perSiteOf(1) * 64 > budget) p.cells = 0;
  const int ncell = p.cells ? p.nc[0] * p.nc[1] * p.nc[2] : 0;
  const long long fixedBytes = fixedOf(p.cells);
  const long long perSite = perSiteOf(p.cells);
  if (fixedBytes + perSite * 64 > budget)
  {
    delete x;
    return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_mixture: the CTA's k-range does not fit in shared memory (use more CTAs)");
  }
  const long long share = (static_cast<long long>(p.capacity) * na + x->blocks - 1) / x->blocks;
  p.nslice = static_cast<int>(std::max<long long>(64, std::min(std::min(share, (budget - fixedBytes) / perSite), 65535ll)));
  x->smem = dynBytes(p.tabK, p.ncand_max, p.cand_atoms, p.kpc, p.nseg_max, p.nslice, ncell);
  err = cudaFuncSetAttribute(p.quintic ? mixtureKernel<true> : mixtureKernel<false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(x->smem));
  if (err == cudaSuccess)
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, p.quintic ? mixtureKernel<true> : mixtureKernel<false>,
                                                        kThreads, x->smem);
  if (err != cudaSuccess || perSM < 1)
  {
    delete x;
    return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_mixture: kernel does not fit on an SM");
  }
  // device state
  const int cap = p.capacity;
  auto alloc = [&](void** ptr, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
    if (err == cudaSuccess) x->allocs.push_back(*ptr);
  };
  float4* dljf = nullptr;
  float* dq = nullptr;
  alloc(reinterpret_cast<void**>(&dljf), sizeof(float4) * ljf.size());
  alloc(reinterpret_cast<void**>(&dq), sizeof(float) * qtype.size());
  alloc(reinterpret_cast<void**>(&x->st.pos), sizeof(double4) * cap * na);
  alloc(reinterpret_cast<void**>(&x->st.fx), sizeof(int4) * cap * na);
  alloc(reinterpret_cast<void**>(&x->st.comp_of), sizeof(int) * cap);
  alloc(reinterpret_cast<void**>(&x->st.list), sizeof(int) * cap * kMaxComp);
  alloc(reinterpret_cast<void**>(&x->st.slot), sizeof(int) * cap);
  alloc(reinterpret_cast<void**>(&x->st.n_state), sizeof(int) * (1 + kMaxComp));
  alloc(reinterpret_cast<void**>(&x->st.energy), sizeof(double));
  alloc(reinterpret_cast<void**>(&x->st.move_base), sizeof(long long));
  alloc(reinterpret_cast<void**>(&x->st.stats), sizeof(double) * kStats);
  alloc(reinterpret_cast<void**>(&x->st.sk), sizeof(double2) * std::max(1, p.nk));
  alloc(reinterpret_cast<void**>(&x->st.part), sizeof(double) * kRow * 2 * x->blocks);
  alloc(reinterpret_cast<void**>(&x->st.bar), sizeof(unsigned long long) * 2);
  alloc(reinterpret_cast<void**>(&x->d_st), sizeof(State));
  int4* dfwx = nullptr;
  float* dfwq = nullptr;
  alloc(reinterpret_cast<void**>(&dfwx), sizeof(int4) * hfw.size());
  alloc(reinterpret_cast<void**>(&dfwq), sizeof(float) * hfq.size());
  x->st.fwx = dfwx;
  x->st.fwq = dfwq;
  x->st.ljf = dljf;
  x->st.qtype = dq;
  // host copies of the starting configuration
  std::vector<double4> hpos(static_cast<size_t>(cap) * na);
  std::vector<int4> hfx(static_cast<size_t>(cap) * na);
  std::vector<int> hcomp(cap, 0), hlist(static_cast<size_t>(cap) * kMaxComp, 0), hslot(cap, 0);
  int counts[kMaxComp] = {0, 0, 0, 0};
  for (int m = 0; m < n_molecules; ++m)
  {
    const int c = comp_of_molecule[m];
    if (c < 0 || c >= n_components)
    {
      freeAll(x);
      delete x;
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture: component index");
    }
    hcomp[m] = c;
    hslot[m] = counts[c];
    hlist[static_cast<size_t>(c) * cap + counts[c]] = m;
    counts[c] += 1;
    // every molecule is stored whole (atom i = atom 0 + the minimum image of their separation), as the reference keeps
    // molecules: a molecule split by per-atom wrapping would have a wrong centre of mass in a rotation
    const double* r0 = xyz + 3 * (static_cast<size_t>(m) * na);
    for (int i = 0; i < na; ++i)
    {
      const double* ri = xyz + 3 * (static_cast<size_t>(m) * na + i);
      double dr[3] = {ri[0] - r0[0], ri[1] - r0[1], ri[2] - r0[2]};
      double sd[3];
      for (int a = 0; a < 3; ++a)
      {
        sd[a] = box.ic[0][a] * dr[0] + box.ic[1][a] * dr[1] + box.ic[2][a] * dr[2];
        sd[a] -= std::nearbyint(sd[a]);
      }
      const double r[3] = {r0[0] + box.c[0][0] * sd[0] + box.c[1][0] * sd[1] + box.c[2][0] * sd[2],
                           r0[1] + box.c[0][1] * sd[0] + box.c[1][1] * sd[1] + box.c[2][1] * sd[2],
                           r0[2] + box.c[0][2] * sd[0] + box.c[1][2] * sd[1] + box.c[2][2] * sd[2]};
      hpos[m * na + i] = make_double4(r[0], r[1], r[2], 0.0);
      double s[3];
      for (int a = 0; a < 3; ++a) s[a] = box.ic[0][a] * r[0] + box.ic[1][a] * r[1] + box.ic[2][a] * r[2];
      int f[3];
      for (int a = 0; a < 3; ++a)
      {
        const double v = s[a] - std::floor(s[a]);
        f[a] = static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(v * 4294967296.0)));
      }
      hfx[m * na + i] = make_int4(f[0], f[1], f[2], comps[c].types[i] | (m << 8));
    }
  }
  int nstate[1 + kMaxComp] = {n_molecules, counts[0], counts[1], counts[2], counts[3]};
  const double zero = 0.0;
  const long long zl = 0;
  cudaStream_t sm = ctx->stream;
  if (err == cudaSuccess) err = cudaMemcpyAsync(dljf, ljf.data(), sizeof(float4) * ljf.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(dq, qtype.data(), sizeof(float) * qtype.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess && !hfw.empty())
    err = cudaMemcpyAsync(dfwx, hfw.data(), sizeof(int4) * hfw.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess && !hfq.empty())
    err = cudaMemcpyAsync(dfwq, hfq.data(), sizeof(float) * hfq.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(x->st.pos, hpos.data(), sizeof(double4) * hpos.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(x->st.fx, hfx.data(), sizeof(int4) * hfx.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(x->st.comp_of, hcomp.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(x->st.list, hlist.data(), sizeof(int) * hlist.size(), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(x->st.slot, hslot.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(x->st.n_state, nstate, sizeof(nstate), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(x->st.energy, &zero, sizeof(double), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemcpyAsync(x->st.move_base, &zl, sizeof(long long), cudaMemcpyHostToDevice, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(x->st.stats, 0, sizeof(double) * kStats, sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(x->st.sk, 0, sizeof(double2) * std::max(1, p.nk), sm);
  if (err == cudaSuccess) err = cudaMemsetAsync(x->st.bar, 0, sizeof(unsigned long long) * 2, sm);
  x->st.spin_limit = kSpinLimit;
  x->st.absent_cta = -1;
  if (err == cudaSuccess) err = cudaStreamSynchronize(sm);
  if (err != cudaSuccess)
  {
    freeAll(x);
    delete x;
    return rg::cudaFail(ctx, err, "rg_mixture_create");
  }
  *out = x;
  return RG_OK;
}

extern "C" rg_status rg_mixture_destroy(rg_mixture* x)
{
  if (!x) return RG_OK;
  cudaSetDevice(x->ctx->device);
  cudaStreamSynchronize(x->ctx->stream);
  freeAll(x);
  delete x;
  return RG_OK;
}

extern "C" rg_status rg_mixture_set_state(rg_mixture* x, double energy, const double* sk, int64_t n_doubles)
{
  if (!x) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = x->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (sk)
  {
    if (n_doubles != 2ll * x->p.nk) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_set_state: 2 nk doubles");
    RG_CUDA(ctx, cudaMemcpyAsync(x->st.sk, sk, sizeof(double) * n_doubles, cudaMemcpyHostToDevice, ctx->stream));
  }
  RG_CUDA(ctx, cudaMemcpyAsync(x->st.energy, &energy, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

extern "C" rg_status rg_mixture_run_many(rg_mixture* const* mixtures, int n, int64_t moves, int record)
{
  if (!mixtures || n < 1 || moves < 0) return RG_ERR_INVALID_ARGUMENT;
  for (int s = 0; s < n; ++s)
    if (!mixtures[s]) return RG_ERR_INVALID_ARGUMENT;
  rg_mixture* x0 = mixtures[0];
  rg_ctx* ctx = x0->ctx;
  if (n > kMaxSystems) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_run_many: at most 148 systems");
  size_t smem = 0;
  for (int s = 0; s < n; ++s)
  {
    if (mixtures[s]->ctx != ctx || mixtures[s]->blocks != x0->blocks)
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_run_many: one context and one CTA count for all");
    // the systems of one launch share everything but their state: same system, Ewald state, components and
    // parameters (their molecules, seeds and statistics may differ)
    if (std::memcmp(&mixtures[s]->p, &x0->p, sizeof(Params)) != 0)
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT,
                      "rg_mixture_run_many: the systems differ in more than their state (system, components, parameters)");
    for (int t = 0; t < s; ++t)
      if (mixtures[t] == mixtures[s])
        return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_run_many: a system listed twice");
    smem = std::max(smem, mixtures[s]->smem);
  }
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  // every system's CTAs must be resident together with the others' (one cooperative launch)
  int sms = 0, perSM = 0;
  RG_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  auto kernel = x0->p.quintic ? mixtureKernel<true> : mixtureKernel<false>;
  RG_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  RG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, kThreads, smem));
  if (static_cast<long long>(n) * x0->blocks > static_cast<long long>(sms) * perSM)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_run_many: the systems' CTAs do not fit on the GPU at once");
  Launch L{};
  L.p = x0->p;
  for (int s = 0; s < n; ++s)
  {
    mixtures[s]->st.record = record ? 1 : 0;
    RG_CUDA(ctx, cudaMemcpyAsync(mixtures[s]->d_st, &mixtures[s]->st, sizeof(State), cudaMemcpyHostToDevice,
                                 ctx->stream));
    L.st[s] = mixtures[s]->d_st;
  }
  const int64_t per = 8192;
  for (int64_t done = 0; done < moves; done += per)
  {
    int m = static_cast<int>(std::min<int64_t>(per, moves - done));
    void* args[] = {&L, &m};
    // every barrier's arrival counter starts at zero in every launch (the error flags beside them persist)
    for (int s = 0; s < n; ++s)
      RG_CUDA(ctx, cudaMemsetAsync(mixtures[s]->st.bar, 0, sizeof(unsigned long long), ctx->stream));
    RG_CUDA(ctx, cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kernel), dim3(n * x0->blocks),
                                             dim3(kThreads), args, smem, ctx->stream));
  }
  return RG_OK;
}

extern "C" rg_status rg_mixture_run(rg_mixture* x, int64_t moves, int record)
{
  if (!x) return RG_ERR_INVALID_ARGUMENT;
  return rg_mixture_run_many(&x, 1, moves, record);
}

extern "C" rg_status rg_mixture_set_wait_test(rg_mixture* x, int absent_cta, int64_t spin_limit)
{
  if (!x || absent_cta < -1 || absent_cta >= x->blocks || spin_limit < 1) return RG_ERR_INVALID_ARGUMENT;
  x->st.absent_cta = absent_cta;
  x->st.spin_limit = std::min<long long>(spin_limit, kSpinLimit);  // never longer than the production limit
  return RG_OK;
}

extern "C" rg_status rg_mixture_results(rg_mixture* x, rg_mixture_result* out)
{
  if (!x || !out) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = x->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  int ns[1 + kMaxComp];
  double e, st[kStats];
  unsigned long long bar[2];
  RG_CUDA(ctx, cudaMemcpyAsync(ns, x->st.n_state, sizeof(ns), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(&e, x->st.energy, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(st, x->st.stats, sizeof(st), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(bar, x->st.bar, sizeof(bar), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memset(out, 0, sizeof(*out));
  for (int c = 0; c < kMaxComp; ++c)
  {
    out->n_molecules[c] = ns[1 + c];
    out->sum_n[c] = st[10 + c];
  }
  out->energy = e;
  for (int k = 0; k < 5; ++k)
  {
    out->attempted[k] = static_cast<int64_t>(st[k]);
    out->accepted[k] = static_cast<int64_t>(st[5 + k]);
  }
  out->sum_energy = st[14];
  out->samples = static_cast<int64_t>(st[15]);
  out->status = bar[1] ? RG_ERR_TIMEOUT : RG_OK;
  return RG_OK;
}

extern "C" rg_status rg_mixture_get_positions(rg_mixture* x, double* xyz, int32_t* comp, int capacity_molecules,
                                              int* n_molecules)
{
  if (!x || !xyz || !comp || !n_molecules) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = x->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  int n = 0;
  RG_CUDA(ctx, cudaMemcpyAsync(&n, x->st.n_state, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (n > capacity_molecules) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_get_positions: capacity");
  std::vector<double4> pos(static_cast<size_t>(n) * x->p.na);
  if (n > 0)
  {
    RG_CUDA(ctx, cudaMemcpyAsync(pos.data(), x->st.pos, sizeof(double4) * pos.size(), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    RG_CUDA(ctx, cudaMemcpyAsync(comp, x->st.comp_of, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
  }
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (size_t i = 0; i < pos.size(); ++i)
  {
    xyz[3 * i] = pos[i].x;
    xyz[3 * i + 1] = pos[i].y;
    xyz[3 * i + 2] = pos[i].z;
  }
  *n_molecules = n;
  return RG_OK;
}

extern "C" rg_status rg_mixture_get_structure_factors(rg_mixture* x, double* host, int64_t n_doubles)
{
  if (!x || !host || n_doubles != 2ll * x->p.nk) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = x->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  RG_CUDA(ctx, cudaMemcpyAsync(host, x->st.sk, sizeof(double) * n_doubles, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

extern "C" rg_status rg_mixture_set_proposal(rg_mixture* x, int component, rg_proposal* proposal,
                                             const rg_box* unit_cell)
{
  if (!x || component < 0 || component >= x->n_comp) return RG_ERR_INVALID_ARGUMENT;
  Comp& c = x->p.comp[component];
  if (!proposal)
  {
    c.prop_cdf = nullptr;
    c.prop_q = nullptr;
    return RG_OK;
  }
  if (!unit_cell) return RG_ERR_INVALID_ARGUMENT;
  rg_status st = rgd::proposalExport(proposal, &c.prop_cdf, &c.prop_q, &c.prop_G, &c.prop_eps);
  if (st) return st;
  // the simulation box must be rep[0] x rep[1] x rep[2] unit cells
  const rg::HostBox ub = rg::makeHostBox(unit_cell);
  for (int a = 0; a < 3; ++a)
  {
    double ratio = 0.0, norm = 0.0;
    for (int r = 0; r < 3; ++r)
    {
      ratio += x->p.box.c[a][r] * ub.c[a][r];
      norm += ub.c[a][r] * ub.c[a][r];
    }
    const double rep = ratio / norm;
    x->p.rep[a] = static_cast<int>(std::lround(rep));
    if (x->p.rep[a] < 1 || std::fabs(rep - x->p.rep[a]) > 1e-9 * rep)
    {
      c.prop_cdf = nullptr;
      c.prop_q = nullptr;
      return rg::fail(x->ctx, RG_ERR_INVALID_ARGUMENT, "rg_mixture_set_proposal: box is not a replication of the cell");
    }
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      x->p.uc[i][j] = ub.c[i][j];
      x->p.uic[i][j] = ub.ic[i][j];
    }
  return RG_OK;
}

extern "C" rg_status rg_mixture_info(rg_mixture* x, int* blocks, int64_t* nk)
{
  if (!x) return RG_ERR_INVALID_ARGUMENT;
  if (blocks) *blocks = x->blocks;
  if (nk) *nk = x->p.nk;
  return RG_OK;
}

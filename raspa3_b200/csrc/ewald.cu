// (c) Ewald Fourier energy of a Monte Carlo move, on device-resident structure factors.
//
// Replaces Interactions::energyDifferenceEwaldFourier (src/raspakit/interactions/ewald.cpp:1043-1244),
// Interactions::acceptEwaldMove (ewald.cpp:1565-1574), Interactions::computeEwaldFourierEnergy (ewald.cpp:352-563)
// and Interactions::precomputeEwaldFourierRigid (ewald.cpp:276-348).
//
// Layout in HBM, per system: the accepted k-vectors in the reference loop order (kx in [0,kmax], ky and kz in
// [-kmax,kmax], k != 0, integer-sphere and reciprocal-cutoff tests) as char4 (kx,ky,kz,-), the prefactor
// temp(k) = C*2pi/V*(kx==0 ? 1 : 2)*exp(-|k|^2/(4 alpha^2))/|k|^2 in FP64, and two FP64 complex structure-factor
// buffers of (1 + groups) entries per k (the total and the dU/dlambda group sums), "stored" and "trial". A move
// writes trial = stored + Delta rho; accepting swaps the two pointers instead of the reference's full vector copy.
// The Fourier energy change per k is computed as temp*(2 Re(conj(S) dRho) + |dRho|^2), algebraically the reference's
// temp*(|S + dRho|^2 - |S|^2) without the cancellation. Block partial sums are reduced in a fixed order by the last
// block to finish (deterministic), which writes the totals straight into mapped pinned host memory. A move of up to 16
// atoms travels in the launch's parameter block, so one difference costs one launch and one synchronisation. The full
// recompute splits the atoms into chunks along a second grid dimension and sums the chunks' partial structure factors
// in chunk order. Self, exclusion and net-charge terms are few-atom FP64 host sums.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"

struct rg_ewald
{
  rg_ctx* ctx = nullptr;
  int n_groups = 0;
  int64_t nk = 0;
  double single_ion_sum = 0.0;  // sum_k temp(k)
  double alpha = 0.0;
  double volume = 0.0;
  rg::HostBox box{};
  rg_forcefield ff{};
  bool omit_inter = false;
  bool use_charge = true;
  // device
  char4* kvec = nullptr;
  double* temp = nullptr;
  double2* s_rigid = nullptr;  // framework structure factor, nk entries (zero if no framework)
  double2* stored = nullptr;   // nk*(1+G)
  double2* trial = nullptr;    // nk*(1+G)
  double* partial = nullptr;   // per-block partial sums
  unsigned int* counter = nullptr;
  double* result = nullptr;    // 1 + G doubles (+ spare): device view of result_host (mapped pinned memory)
  double2* scratch = nullptr;  // full recompute: partial structure factors per atom chunk
  size_t scratch_bytes = 0;
  int sms = 148;
  void* moved = nullptr;       // moved-atom staging (device)
  size_t moved_bytes = 0;
  void* moved_host = nullptr;  // pinned staging
  double* result_host = nullptr;  // mapped pinned: the kernels' last block writes the totals here directly
};

namespace
{
constexpr int kThreads = 256;
constexpr int kMaxGroups = 4;
constexpr int kMaxMoved = 512;  // old + new atoms of one move (staged in shared memory)
constexpr int kParamMoved = 16; // moves of up to this many atoms travel in the launch's parameter block

struct MovedAtom
{
  double s[3];   // fractional coordinates (inverse cell * position)
  double w;      // sign * scalingCoulomb * charge (sign -1 for old atoms)
  double wg;     // sign * charge (dU/dlambda group sums)
  int group;     // 0 = none, 1..4
  int pad;
};

// the moved atoms of a small move, passed by value in the launch parameters (no copy before the launch)
struct MovedParam
{
  MovedAtom a[kParamMoved];
};

__device__ __forceinline__ double2 phase(const char4 k, const double* s)
{
  // exp(i 2 pi k.s)
  double arg = 2.0 * (static_cast<double>(k.x) * s[0] + static_cast<double>(k.y) * s[1] +
                      static_cast<double>(k.z) * s[2]);
  double sn, cs;
  sincospi(arg, &sn, &cs);
  return make_double2(cs, sn);
}

template <int G>
__device__ __forceinline__ void blockReduceAndFinish(double (&v)[1 + G], double* partial, unsigned int* counter,
                                                     double* result)
{
  __shared__ double red[kThreads / 32][1 + kMaxGroups];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 1 + G; ++c)
  {
    double x = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][c] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    for (int c = 0; c < 1 + G; ++c)
    {
      double x = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) x += red[w][c];
      partial[blockIdx.x * (1 + kMaxGroups) + c] = x;
    }
    __threadfence();
    unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block: each thread sums the partials of blocks threadIdx.x, threadIdx.x + blockDim.x, ... (all its loads
  // in flight together), then the same fixed-order warp and block reduction
  double y[1 + G];
#pragma unroll
  for (int c = 0; c < 1 + G; ++c) y[c] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
  {
#pragma unroll
    for (int c = 0; c < 1 + G; ++c) y[c] += __ldcg(partial + b * (1 + kMaxGroups) + c);
  }
#pragma unroll
  for (int c = 0; c < 1 + G; ++c)
  {
    double x = y[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][c] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    for (int c = 0; c < 1 + G; ++c)
    {
      double x = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) x += red[w][c];
      result[c] = x;
    }
    *counter = 0u;  // ready for the next launch on this system
  }
}

// One thread per k-vector: the change of the structure factor caused by the moved atoms, the Fourier energy change
// and its dU/dlambda group terms, and the trial structure factor.
template <int G>
__global__ void __launch_bounds__(kThreads) ewaldDeltaKernel(int64_t nk, const char4* __restrict__ kvec,
                                                             const double* __restrict__ temp,
                                                             const double2* __restrict__ stored,
                                                             double2* __restrict__ trial,
                                                             const MovedAtom* __restrict__ moved, MovedParam small,
                                                             int n_moved, double* partial, unsigned int* counter,
                                                             double* result)
{
  extern __shared__ MovedAtom sm[];
  for (int a = threadIdx.x; a < n_moved; a += blockDim.x) sm[a] = moved ? moved[a] : small.a[a];
  __syncthreads();
  double v[1 + G];
#pragma unroll
  for (int c = 0; c < 1 + G; ++c) v[c] = 0.0;
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < nk)
  {
    const char4 kv = kvec[k];
    double2 d = make_double2(0.0, 0.0);
    double2 dg[G > 0 ? G : 1];
#pragma unroll
    for (int g = 0; g < (G > 0 ? G : 1); ++g) dg[g] = make_double2(0.0, 0.0);
    for (int a = 0; a < n_moved; ++a)
    {
      double2 e = phase(kv, sm[a].s);
      d.x += sm[a].w * e.x;
      d.y += sm[a].w * e.y;
      if (G > 0)
      {
        int g = sm[a].group;
#pragma unroll
        for (int gg = 0; gg < (G > 0 ? G : 1); ++gg)
          if (g == gg + 1)
          {
            dg[gg].x += sm[a].wg * e.x;
            dg[gg].y += sm[a].wg * e.y;
          }
      }
    }
    const double t = temp[k];
    const double2 S = stored[k * (1 + G)];
    const double2 T = make_double2(S.x + d.x, S.y + d.y);
    v[0] = t * (2.0 * (S.x * d.x + S.y * d.y) + (d.x * d.x + d.y * d.y));
    trial[k * (1 + G)] = T;
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      const double2 SG = stored[k * (1 + G) + 1 + g];
      const double2 TG = make_double2(SG.x + dg[g].x, SG.y + dg[g].y);
      // addFourierDUdlambda(2 temp, T, TG) - addFourierDUdlambda(2 temp, S, SG)  (ewald.cpp:166-173)
      v[1 + g] = 2.0 * t * ((T.x * TG.x + T.y * TG.y) - (S.x * SG.x + S.y * SG.y));
      trial[k * (1 + G) + 1 + g] = TG;
    }
  }
  blockReduceAndFinish<G>(v, partial, counter, result);
}

// Per-atom phase tables for the full structure factor: e^{i 2 pi m s_d}, m = 0..kmax_d, built in shared memory for
// a tile of atoms; each thread owns one k-vector and accumulates over the tile with two complex products per atom.
constexpr int kFullTile = 32;

template <int G>
__global__ void __launch_bounds__(kThreads) ewaldFullPartialKernel(int64_t nk, const char4* __restrict__ kvec,
                                                                   const MovedAtom* __restrict__ atoms, int n_atoms,
                                                                   int chunk_atoms, int kxm, int kym, int kzm,
                                                                   double2* __restrict__ scratch)
{
  // blockIdx.y: a chunk of atoms; each thread owns one k-vector and sums the chunk's atoms with two complex products
  // per atom, from per-atom phase tables e^{i 2 pi m s_d} (m = 0..kmax_d) built in shared memory per tile
  extern __shared__ double2 tab[];  // kFullTile * (kxm+1 + kym+1 + kzm+1)
  __shared__ double wq[kFullTile], wgq[kFullTile];
  __shared__ int grp[kFullTile];
  const int stride = (kxm + 1) + (kym + 1) + (kzm + 1);
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int a0 = blockIdx.y * chunk_atoms, a1 = min(n_atoms, a0 + chunk_atoms);
  char4 kv = make_char4(0, 0, 0, 0);
  if (k < nk) kv = kvec[k];
  double2 acc = make_double2(0.0, 0.0);
  double2 accg[G > 0 ? G : 1];
#pragma unroll
  for (int g = 0; g < (G > 0 ? G : 1); ++g) accg[g] = make_double2(0.0, 0.0);
  for (int base = a0; base < a1; base += kFullTile)
  {
    const int na = min(kFullTile, a1 - base);
    __syncthreads();
    for (int idx = threadIdx.x; idx < na * stride; idx += blockDim.x)
    {
      int a = idx / stride, m = idx % stride;
      int d = (m <= kxm) ? 0 : ((m <= kxm + 1 + kym) ? 1 : 2);
      int mm = (d == 0) ? m : ((d == 1) ? m - (kxm + 1) : m - (kxm + 1) - (kym + 1));
      double sn, cs;
      sincospi(2.0 * static_cast<double>(mm) * atoms[base + a].s[d], &sn, &cs);
      tab[a * stride + m] = make_double2(cs, sn);
    }
    for (int a = threadIdx.x; a < na; a += blockDim.x)
    {
      wq[a] = atoms[base + a].w;
      wgq[a] = atoms[base + a].wg;
      grp[a] = atoms[base + a].group;
    }
    __syncthreads();
    if (k < nk)
    {
      const int ax = kv.x, ay = abs(kv.y), az = abs(kv.z);
      const double sy = kv.y < 0 ? -1.0 : 1.0, sz = kv.z < 0 ? -1.0 : 1.0;
      for (int a = 0; a < na; ++a)
      {
        const double2* t = tab + a * stride;
        double2 ex = t[ax], ey = t[kxm + 1 + ay], ez = t[kxm + 1 + kym + 1 + az];
        ey.y *= sy;
        ez.y *= sz;
        double2 xy = make_double2(ex.x * ey.x - ex.y * ey.y, ex.x * ey.y + ex.y * ey.x);
        double2 e = make_double2(xy.x * ez.x - xy.y * ez.y, xy.x * ez.y + xy.y * ez.x);
        acc.x += wq[a] * e.x;
        acc.y += wq[a] * e.y;
        if (G > 0)
        {
#pragma unroll
          for (int gg = 0; gg < (G > 0 ? G : 1); ++gg)
            if (grp[a] == gg + 1)
            {
              accg[gg].x += wgq[a] * e.x;
              accg[gg].y += wgq[a] * e.y;
            }
        }
      }
    }
  }
  if (k < nk)
  {
    double2* out = scratch + (static_cast<int64_t>(blockIdx.y) * nk + k) * (1 + G);
    out[0] = acc;
#pragma unroll
    for (int g = 0; g < G; ++g) out[1 + g] = accg[g];
  }
}

// The chunks' partial structure factors summed in chunk order, the framework's added, the Fourier energy and its
// dU/dlambda group terms (ewald.cpp:458-468), reduced in a fixed order by the last block.
template <int G>
__global__ void __launch_bounds__(kThreads) ewaldFullFinishKernel(int64_t nk, int n_chunks,
                                                                  const double2* __restrict__ scratch,
                                                                  const double* __restrict__ temp,
                                                                  const double2* __restrict__ s_rigid,
                                                                  double2* __restrict__ stored, int omit_inter,
                                                                  double* partial, unsigned int* counter,
                                                                  double* result)
{
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  double v[1 + G];
#pragma unroll
  for (int c = 0; c < 1 + G; ++c) v[c] = 0.0;
  if (k < nk)
  {
    double2 acc = make_double2(0.0, 0.0);
    double2 accg[G > 0 ? G : 1];
#pragma unroll
    for (int g = 0; g < (G > 0 ? G : 1); ++g) accg[g] = make_double2(0.0, 0.0);
    for (int c = 0; c < n_chunks; ++c)
    {
      const double2* in = scratch + (static_cast<int64_t>(c) * nk + k) * (1 + G);
      acc.x += in[0].x;
      acc.y += in[0].y;
#pragma unroll
      for (int g = 0; g < G; ++g)
      {
        accg[g].x += in[1 + g].x;
        accg[g].y += in[1 + g].y;
      }
    }
    const double t = temp[k];
    const double2 R = s_rigid[k];
    const double2 T = make_double2(R.x + acc.x, R.y + acc.y);
    // temp*(|S_fw + S_ads|^2 - |S_fw|^2) = temp*(2 Re(conj(S_fw) S_ads) + |S_ads|^2)  (ewald.cpp:458-468)
    v[0] = t * (2.0 * (R.x * acc.x + R.y * acc.y) + (acc.x * acc.x + acc.y * acc.y));
    if (omit_inter) v[0] -= t * (acc.x * acc.x + acc.y * acc.y);
    stored[k * (1 + G)] = T;
#pragma unroll
    for (int g = 0; g < G; ++g)
    {
      // rigid group sums are zero (precomputeEwaldFourierRigid sets only the total)
      v[1 + g] = 2.0 * t * (T.x * accg[g].x + T.y * accg[g].y);
      stored[k * (1 + G) + 1 + g] = accg[g];
    }
  }
  blockReduceAndFinish<G>(v, partial, counter, result);
}

// Framework structure factor: the same accumulation without energy terms.
__global__ void __launch_bounds__(kThreads) ewaldRigidKernel(int64_t nk, const char4* __restrict__ kvec,
                                                             double2* __restrict__ s_rigid,
                                                             const MovedAtom* __restrict__ atoms, int n_atoms, int kxm,
                                                             int kym, int kzm)
{
  extern __shared__ double2 tab[];
  __shared__ double wq[kFullTile];
  const int stride = (kxm + 1) + (kym + 1) + (kzm + 1);
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  char4 kv = make_char4(0, 0, 0, 0);
  if (k < nk) kv = kvec[k];
  double2 acc = make_double2(0.0, 0.0);
  for (int base = 0; base < n_atoms; base += kFullTile)
  {
    const int na = min(kFullTile, n_atoms - base);
    __syncthreads();
    for (int idx = threadIdx.x; idx < na * stride; idx += blockDim.x)
    {
      int a = idx / stride, m = idx % stride;
      int d = (m <= kxm) ? 0 : ((m <= kxm + 1 + kym) ? 1 : 2);
      int mm = (d == 0) ? m : ((d == 1) ? m - (kxm + 1) : m - (kxm + 1) - (kym + 1));
      double sn, cs;
      sincospi(2.0 * static_cast<double>(mm) * atoms[base + a].s[d], &sn, &cs);
      tab[a * stride + m] = make_double2(cs, sn);
    }
    for (int a = threadIdx.x; a < na; a += blockDim.x) wq[a] = atoms[base + a].w;
    __syncthreads();
    if (k < nk)
    {
      const int ax = kv.x, ay = abs(kv.y), az = abs(kv.z);
      const double sy = kv.y < 0 ? -1.0 : 1.0, sz = kv.z < 0 ? -1.0 : 1.0;
      for (int a = 0; a < na; ++a)
      {
        const double2* t = tab + a * stride;
        double2 ex = t[ax], ey = t[kxm + 1 + ay], ez = t[kxm + 1 + kym + 1 + az];
        ey.y *= sy;
        ez.y *= sz;
        double2 xy = make_double2(ex.x * ey.x - ex.y * ey.y, ex.x * ey.y + ex.y * ey.x);
        double2 e = make_double2(xy.x * ez.x - xy.y * ez.y, xy.x * ez.y + xy.y * ez.x);
        acc.x += wq[a] * e.x;
        acc.y += wq[a] * e.y;
      }
    }
  }
  if (k < nk) s_rigid[k] = acc;
}

inline int groupOf(const rg_atom& a) { return a.group_fractional & 0x0f; }

void roundHalfAwayPbc(const rg::HostBox& b, double dr[3])
{
  // SimulationBox::applyPeriodicBoundaryConditions (src/raspakit/simulationbox.ixx:131-161)
  auto rnd = [](double x) { return static_cast<double>(static_cast<long long>(x + ((x >= 0.0) ? 0.5 : -0.5))); };
  if (!b.triclinic)
  {
    dr[0] -= rnd(dr[0] * b.ic[0][0]) * b.c[0][0];
    dr[1] -= rnd(dr[1] * b.ic[1][1]) * b.c[1][1];
    dr[2] -= rnd(dr[2] * b.ic[2][2]) * b.c[2][2];
    return;
  }
  double s[3];
  rg::matvec(b.ic, dr, s);
  for (int d = 0; d < 3; ++d) s[d] -= rnd(s[d]);
  rg::matvec(b.c, s, dr);
}

// Potentials::ewaldExclusionFactors (src/raspakit/potentials/coulomb_real_space.ixx:49-65)
void exclusionFactors(double alpha, double scalingTotal, double r, double& potential, double& dudl)
{
  const double s = r + 0.01 * (1.0 - scalingTotal);
  const double inverseS = 1.0 / s;
  potential = std::erf(alpha * s) * inverseS;
  const double gaussianTerm = 2.0 * alpha * rg::kInvSqrtPi * std::exp(-alpha * alpha * s * s);
  const double firstDerivative = (gaussianTerm - potential) * inverseS;
  dudl = potential - scalingTotal * 0.01 * firstDerivative;
}

void addDud(double* arr, int gA, int gB, double sA, double sB, double factor)
{
  if (gA != 0) arr[gA - 1] += sB * factor;
  if (gB != 0) arr[gB - 1] += sA * factor;
}

// fractional coordinates and signed weights of the old (sign old_sign) and new atoms of a move
void packMoved(const rg_ewald* e, const rg_atom* old_atoms, int n_old, const rg_atom* new_atoms, int n_new,
               double old_sign, MovedAtom* h)
{
  for (int i = 0; i < n_old + n_new; ++i)
  {
    const bool isOld = i < n_old;
    const rg_atom& a = isOld ? old_atoms[i] : new_atoms[i - n_old];
    const double sign = isOld ? old_sign : 1.0;
    double r[3] = {a.x, a.y, a.z};
    rg::matvec(e->box.ic, r, h[i].s);
    h[i].w = sign * a.scaling_coulomb * a.charge;
    h[i].wg = sign * a.charge;
    h[i].group = groupOf(a);
    h[i].pad = 0;
  }
}

rg_status stageAtoms(rg_ewald* e, const rg_atom* old_atoms, int n_old, const rg_atom* new_atoms, int n_new,
                     double old_sign)
{
  rg_ctx* ctx = e->ctx;
  const int n = n_old + n_new;
  const size_t bytes = sizeof(MovedAtom) * static_cast<size_t>(n > 0 ? n : 1);
  if (e->moved_bytes < bytes)
  {
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (e->moved) cudaFree(e->moved);
    if (e->moved_host) cudaFreeHost(e->moved_host);
    size_t grow = bytes * 2;
    RG_CUDA(ctx, cudaMalloc(&e->moved, grow));
    RG_CUDA(ctx, cudaMallocHost(&e->moved_host, grow));
    e->moved_bytes = grow;
  }
  else
  {
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the staging buffer of the previous call is free again
  }
  MovedAtom* h = static_cast<MovedAtom*>(e->moved_host);
  packMoved(e, old_atoms, n_old, new_atoms, n_new, old_sign, h);
  if (n > 0) RG_CUDA(ctx, cudaMemcpyAsync(e->moved, h, sizeof(MovedAtom) * n, cudaMemcpyHostToDevice, ctx->stream));
  return RG_OK;
}

template <int G>
cudaError_t launchDelta(rg_ewald* e, int n_moved, const MovedParam* small)
{
  const int blocks = static_cast<int>((e->nk + kThreads - 1) / kThreads);
  ewaldDeltaKernel<G><<<blocks, kThreads, sizeof(MovedAtom) * (n_moved > 0 ? n_moved : 1), e->ctx->stream>>>(
      e->nk, e->kvec, e->temp, e->stored, e->trial, small ? nullptr : static_cast<const MovedAtom*>(e->moved),
      small ? *small : MovedParam{}, n_moved, e->partial, e->counter, e->result);
  return cudaGetLastError();
}

template <int G>
cudaError_t launchFull(rg_ewald* e, int n_atoms)
{
  // atoms split into chunks so that k-blocks x chunks fill the GPU (about four CTAs per SM), at least one tile each
  const int blocks = static_cast<int>((e->nk + kThreads - 1) / kThreads);
  const int maxChunks = std::max(1, (n_atoms + kFullTile - 1) / kFullTile);
  const int chunks = std::min(maxChunks, std::max(1, (4 * e->sms + blocks - 1) / blocks));
  const int chunkAtoms = std::max(kFullTile, (((n_atoms + chunks - 1) / chunks + kFullTile - 1) / kFullTile) * kFullTile);
  const int n_chunks = n_atoms > 0 ? (n_atoms + chunkAtoms - 1) / chunkAtoms : 1;
  const size_t need = sizeof(double2) * static_cast<size_t>(n_chunks) * e->nk * (1 + G);
  if (e->scratch_bytes < need)
  {
    cudaError_t err = cudaStreamSynchronize(e->ctx->stream);
    if (err) return err;
    if (e->scratch) cudaFree(e->scratch);
    e->scratch = nullptr;
    e->scratch_bytes = 0;
    err = cudaMalloc(reinterpret_cast<void**>(&e->scratch), need);
    if (err) return err;
    e->scratch_bytes = need;
  }
  const int stride = (e->ff.kmax_x + 1) + (e->ff.kmax_y + 1) + (e->ff.kmax_z + 1);
  size_t shmem = sizeof(double2) * kFullTile * stride;
  auto kern = ewaldFullPartialKernel<G>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shmem));
  if (n_atoms > 0)
    kern<<<dim3(blocks, n_chunks), kThreads, shmem, e->ctx->stream>>>(
        e->nk, e->kvec, static_cast<const MovedAtom*>(e->moved), n_atoms, chunkAtoms, e->ff.kmax_x, e->ff.kmax_y,
        e->ff.kmax_z, e->scratch);
  else
    cudaMemsetAsync(e->scratch, 0, need, e->ctx->stream);
  ewaldFullFinishKernel<G><<<blocks, kThreads, 0, e->ctx->stream>>>(e->nk, n_chunks, e->scratch, e->temp, e->s_rigid,
                                                                    e->stored, e->omit_inter ? 1 : 0, e->partial,
                                                                    e->counter, e->result);
  return cudaGetLastError();
}

rg_status readResult(rg_ewald* e, double* out, int n)
{
  // the last block wrote the totals into mapped pinned memory: the stream's completion makes them visible here
  rg_ctx* ctx = e->ctx;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(out, e->result_host, sizeof(double) * n);
  return RG_OK;
}
}  // namespace

extern "C"
{
rg_status rg_ewald_create(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* box, int n_groups, rg_ewald** out)
{
  if (!ctx || !ff || !box || !out) return RG_ERR_INVALID_ARGUMENT;
  if (n_groups < 0 || n_groups > kMaxGroups) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_create: groups");
  if (ff->kmax_x < 0 || ff->kmax_y < 0 || ff->kmax_z < 0 || ff->kmax_x > 127 || ff->kmax_y > 127 || ff->kmax_z > 127)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_create: kmax must be in [0, 127]");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_ewald* e = new rg_ewald();
  e->ctx = ctx;
  e->n_groups = n_groups;
  e->box = rg::makeHostBox(box);
  e->ff = *ff;
  e->ff.epsilon = e->ff.sigma = e->ff.shift = nullptr;
  e->ff.lj = nullptr;
  e->alpha = ff->ewald_alpha;
  e->volume = e->box.volume;
  e->omit_inter = ff->omit_inter != 0;
  e->use_charge = ff->use_charge != 0;
  // k-vector set and prefactors in the reference order (ewald.cpp:1098-1146)
  std::vector<char4> kv;
  std::vector<double> tp;
  const double ax[3] = {e->box.ic[0][0], e->box.ic[1][0], e->box.ic[2][0]};
  const double ay[3] = {e->box.ic[0][1], e->box.ic[1][1], e->box.ic[2][1]};
  const double az[3] = {e->box.ic[0][2], e->box.ic[1][2], e->box.ic[2][2]};
  const double prefactor = rg::coulombFactor() * (2.0 * rg::kPi / e->volume);
  const double alpha_squared = ff->ewald_alpha * ff->ewald_alpha;
  double sum = 0.0;
  for (int kx = 0; kx <= ff->kmax_x; ++kx)
  {
    const double factor = (kx == 0) ? (1.0 * prefactor) : (2.0 * prefactor);
    for (int ky = -ff->kmax_y; ky <= ff->kmax_y; ++ky)
      for (int kz = -ff->kmax_z; kz <= ff->kmax_z; ++kz)
      {
        double kvv[3];
        for (int d = 0; d < 3; ++d)
          kvv[d] = 2.0 * rg::kPi * kx * ax[d] + 2.0 * rg::kPi * ky * ay[d] + 2.0 * rg::kPi * kz * az[d];
        double rksq = kvv[0] * kvv[0] + kvv[1] * kvv[1] + kvv[2] * kvv[2];
        uint64_t ksq = static_cast<uint64_t>(kx * kx + ky * ky + kz * kz);
        if ((ksq != 0) && (ksq <= ff->recip_int_cutoff_sq) && (rksq < ff->recip_cutoff_sq))
        {
          double t = factor * std::exp((-0.25 / alpha_squared) * rksq) / rksq;
          kv.push_back(make_char4(static_cast<signed char>(kx), static_cast<signed char>(ky),
                                  static_cast<signed char>(kz), 0));
          tp.push_back(t);
          sum += t;
        }
      }
  }
  e->nk = static_cast<int64_t>(kv.size());
  e->single_ion_sum = sum;
  const int64_t nk = e->nk > 0 ? e->nk : 1;
  const int blocks = static_cast<int>((nk + kThreads - 1) / kThreads);
  auto alloc = [&](void** p, size_t b) { return cudaMalloc(p, b); };
  cudaError_t err = cudaSuccess;
  if (!err) err = alloc(reinterpret_cast<void**>(&e->kvec), sizeof(char4) * nk);
  if (!err) err = alloc(reinterpret_cast<void**>(&e->temp), sizeof(double) * nk);
  if (!err) err = alloc(reinterpret_cast<void**>(&e->s_rigid), sizeof(double2) * nk);
  if (!err) err = alloc(reinterpret_cast<void**>(&e->stored), sizeof(double2) * nk * (1 + n_groups));
  if (!err) err = alloc(reinterpret_cast<void**>(&e->trial), sizeof(double2) * nk * (1 + n_groups));
  if (!err) err = alloc(reinterpret_cast<void**>(&e->partial), sizeof(double) * blocks * (1 + kMaxGroups));
  if (!err) err = alloc(reinterpret_cast<void**>(&e->counter), sizeof(unsigned int) * 4);
  if (!err) err = cudaHostAlloc(reinterpret_cast<void**>(&e->result_host), sizeof(double) * 8, cudaHostAllocMapped);
  if (!err) err = cudaHostGetDevicePointer(reinterpret_cast<void**>(&e->result), e->result_host, 0);
  if (!err) err = cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (!err && e->nk > 0)
    err = cudaMemcpyAsync(e->kvec, kv.data(), sizeof(char4) * e->nk, cudaMemcpyHostToDevice, ctx->stream);
  if (!err && e->nk > 0)
    err = cudaMemcpyAsync(e->temp, tp.data(), sizeof(double) * e->nk, cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMemsetAsync(e->s_rigid, 0, sizeof(double2) * nk, ctx->stream);
  if (!err) err = cudaMemsetAsync(e->stored, 0, sizeof(double2) * nk * (1 + n_groups), ctx->stream);
  if (!err) err = cudaMemsetAsync(e->counter, 0, sizeof(unsigned int) * 4, ctx->stream);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (err)
  {
    rg_status st = rg::cudaFail(ctx, err, "rg_ewald_create");
    rg_ewald_destroy(e);
    return st;
  }
  *out = e;
  return RG_OK;
}

rg_status rg_ewald_destroy(rg_ewald* e)
{
  if (!e) return RG_OK;
  if (e->ctx) cudaStreamSynchronize(e->ctx->stream);
  cudaFree(e->kvec);
  cudaFree(e->temp);
  cudaFree(e->s_rigid);
  cudaFree(e->stored);
  cudaFree(e->trial);
  cudaFree(e->partial);
  cudaFree(e->counter);
  if (e->scratch) cudaFree(e->scratch);
  if (e->moved) cudaFree(e->moved);
  if (e->moved_host) cudaFreeHost(e->moved_host);
  if (e->result_host) cudaFreeHost(e->result_host);
  delete e;
  return RG_OK;
}

rg_status rg_ewald_info(rg_ewald* e, int64_t* n_kvectors, double* single_ion_sum)
{
  if (!e) return RG_ERR_INVALID_ARGUMENT;
  if (n_kvectors) *n_kvectors = e->nk;
  if (single_ion_sum) *single_ion_sum = e->single_ion_sum;
  return RG_OK;
}

rg_status rg_ewald_set_framework(rg_ewald* e, const rg_atom* fw, int n_fw)
{
  if (!e || (n_fw > 0 && !fw) || n_fw < 0) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n_fw == 0 || e->nk == 0)
  {
    RG_CUDA(ctx, cudaMemsetAsync(e->s_rigid, 0, sizeof(double2) * (e->nk > 0 ? e->nk : 1), ctx->stream));
    return RG_OK;
  }
  rg_status st = stageAtoms(e, fw, n_fw, nullptr, 0, 1.0);
  if (st) return st;
  const int blocks = static_cast<int>((e->nk + kThreads - 1) / kThreads);
  const int stride = (e->ff.kmax_x + 1) + (e->ff.kmax_y + 1) + (e->ff.kmax_z + 1);
  size_t shmem = sizeof(double2) * kFullTile * stride;
  cudaFuncSetAttribute(ewaldRigidKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shmem));
  ewaldRigidKernel<<<blocks, kThreads, shmem, ctx->stream>>>(e->nk, e->kvec, e->s_rigid,
                                                            static_cast<const MovedAtom*>(e->moved), n_fw,
                                                            e->ff.kmax_x, e->ff.kmax_y, e->ff.kmax_z);
  RG_CUDA(ctx, cudaGetLastError());
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

rg_status rg_ewald_full(rg_ewald* e, const rg_atom* atoms, int n_atoms, const int32_t* molecule_sizes, int n_molecules,
                        double net_charge_framework, rg_ewald_energy* out)
{
  if (!e || !out || (n_atoms > 0 && !atoms) || n_atoms < 0 || (n_molecules > 0 && !molecule_sizes))
    return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  std::memset(out, 0, sizeof(rg_ewald_energy));
  if (rg_status fs = rg::checkFinite(ctx, atoms, n_atoms, "rg_ewald_full")) return fs;
  if (!e->use_charge) return RG_OK;
  if (!e->omit_inter)
  {
    int64_t total = 0;
    for (int m = 0; m < n_molecules; ++m)
    {
      if (molecule_sizes[m] < 0) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_full: molecule sizes");
      total += molecule_sizes[m];
    }
    if (total > n_atoms) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_full: molecule sizes");
  }
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int G = e->n_groups;
  double res[1 + kMaxGroups] = {0, 0, 0, 0, 0};
  if (e->nk > 0)
  {
    rg_status st = stageAtoms(e, nullptr, 0, atoms, n_atoms, 1.0);
    if (st) return st;
    cudaError_t err;
    switch (G)
    {
      case 0: err = launchFull<0>(e, n_atoms); break;
      case 1: err = launchFull<1>(e, n_atoms); break;
      case 2: err = launchFull<2>(e, n_atoms); break;
      case 3: err = launchFull<3>(e, n_atoms); break;
      default: err = launchFull<4>(e, n_atoms); break;
    }
    if (err) return rg::cudaFail(ctx, err, "ewaldFullKernel");
  }
  // the host terms below run while the kernels are in flight; the reciprocal-space sum is read afterwards
  const double C = rg::coulombFactor();
  const double alpha = e->alpha;
  if (!e->omit_inter)
  {
    // self energy and intramolecular exclusion (ewald.cpp:480-524)
    const double prefactor_self = C * alpha / std::sqrt(rg::kPi);
    for (int i = 0; i < n_atoms; ++i)
    {
      const double q = atoms[i].charge, sc = atoms[i].scaling_coulomb;
      const int g = groupOf(atoms[i]);
      out->ewald_self -= prefactor_self * sc * q * sc * q;
      if (g != 0) out->dudlambda_ewald[g - 1] -= 2.0 * prefactor_self * sc * q * q;
    }
    int index = 0;
    for (int m = 0; m < n_molecules; ++m)
    {
      const int size = molecule_sizes[m];
      const rg_atom* span = atoms + index;
      for (int i = 0; i + 1 < size; ++i)
        for (int j = i + 1; j < size; ++j)
        {
          double dr[3] = {span[i].x - span[j].x, span[i].y - span[j].y, span[i].z - span[j].z};
          roundHalfAwayPbc(e->box, dr);
          const double r = std::sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
          const double sA = span[i].scaling_coulomb, sB = span[j].scaling_coulomb;
          double pot, dudl;
          exclusionFactors(alpha, sA * sB, r, pot, dudl);
          const double prefactor = C * span[i].charge * span[j].charge;
          out->ewald_exclusion -= sA * sB * prefactor * pot;
          addDud(out->dudlambda_ewald, groupOf(span[i]), groupOf(span[j]), sA, sB, -prefactor * dudl);
        }
      index += size;
    }
  }
  // net-charge correction (ewald.cpp:526-560)
  double netChargeAdsorbates = 0.0, netChargeDerivative[4] = {0, 0, 0, 0};
  for (int i = 0; i < n_atoms; ++i)
  {
    netChargeAdsorbates += atoms[i].scaling_coulomb * atoms[i].charge;
    const int g = groupOf(atoms[i]);
    if (g != 0) netChargeDerivative[g - 1] += atoms[i].charge;
  }
  const double uIon = -(e->single_ion_sum - C * alpha / std::sqrt(rg::kPi));
  double netFourier = 0.0, netDudl[4] = {0, 0, 0, 0};
  if (e->omit_inter)
  {
    netFourier = 2.0 * uIon * net_charge_framework * netChargeAdsorbates;
    for (int g = 0; g < 4; ++g) netDudl[g] = 2.0 * uIon * net_charge_framework * netChargeDerivative[g];
  }
  else
  {
    netFourier = uIon * (2.0 * net_charge_framework + netChargeAdsorbates) * netChargeAdsorbates;
    for (int g = 0; g < 4; ++g)
      netDudl[g] = 2.0 * uIon * (net_charge_framework + netChargeAdsorbates) * netChargeDerivative[g];
  }
  if (e->nk > 0)
  {
    rg_status st = readResult(e, res, 1 + G);
    if (st) return st;
  }
  out->ewald_fourier = res[0] + netFourier;
  for (int g = 0; g < G; ++g) out->dudlambda_ewald[g] += res[1 + g];
  for (int g = 0; g < 4; ++g) out->dudlambda_ewald[g] += netDudl[g];
  return RG_OK;
}

rg_status rg_ewald_delta(rg_ewald* e, const rg_atom* new_atoms, int n_new, const rg_atom* old_atoms, int n_old,
                         double net_charge, const double* net_charge_derivative_ext, rg_ewald_energy* out)
{
  if (!e || !out || n_new < 0 || n_old < 0 || (n_new > 0 && !new_atoms) || (n_old > 0 && !old_atoms))
    return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  std::memset(out, 0, sizeof(rg_ewald_energy));
  if (rg_status fs = rg::checkFinite(ctx, new_atoms, n_new, "rg_ewald_delta")) return fs;
  if (rg_status fs = rg::checkFinite(ctx, old_atoms, n_old, "rg_ewald_delta")) return fs;
  if (!e->use_charge) return RG_OK;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int G = e->n_groups;
  const int n = n_old + n_new;
  if (n > kMaxMoved) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_delta: at most 512 old + new atoms");
  double res[1 + kMaxGroups] = {0, 0, 0, 0, 0};
  if (e->nk > 0)
  {
    MovedParam small{};
    const bool inParams = n <= kParamMoved;
    if (inParams)
      packMoved(e, old_atoms, n_old, new_atoms, n_new, -1.0, small.a);
    else
    {
      rg_status st = stageAtoms(e, old_atoms, n_old, new_atoms, n_new, -1.0);
      if (st) return st;
    }
    const MovedParam* sp = inParams ? &small : nullptr;
    cudaError_t err;
    switch (G)
    {
      case 0: err = launchDelta<0>(e, n, sp); break;
      case 1: err = launchDelta<1>(e, n, sp); break;
      case 2: err = launchDelta<2>(e, n, sp); break;
      case 3: err = launchDelta<3>(e, n, sp); break;
      default: err = launchDelta<4>(e, n, sp); break;
    }
    if (err) return rg::cudaFail(ctx, err, "ewaldDeltaKernel");
    rg_status st = readResult(e, res, 1 + G);
    if (st) return st;
  }
  out->ewald_fourier = res[0];
  for (int g = 0; g < G; ++g) out->dudlambda_ewald[g] = res[1 + g];
  const double C = rg::coulombFactor();
  const double alpha = e->alpha;
  // intramolecular exclusion (ewald.cpp:1164-1219): old +, new -; pairs matched on moleculeId
  auto exclusion = [&](const rg_atom* atoms, int count, double sign)
  {
    for (int i = 0; i < count; ++i)
      for (int j = i + 1; j < count; ++j)
      {
        if (atoms[i].molecule_id != atoms[j].molecule_id) continue;
        double dr[3] = {atoms[i].x - atoms[j].x, atoms[i].y - atoms[j].y, atoms[i].z - atoms[j].z};
        roundHalfAwayPbc(e->box, dr);
        const double r = std::sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        const double sA = atoms[i].scaling_coulomb, sB = atoms[j].scaling_coulomb;
        double pot, dudl;
        exclusionFactors(alpha, sA * sB, r, pot, dudl);
        const double prefactor = C * atoms[i].charge * atoms[j].charge;
        out->ewald_exclusion += sign * sA * sB * prefactor * pot;
        addDud(out->dudlambda_ewald, groupOf(atoms[i]), groupOf(atoms[j]), sA, sB, sign * prefactor * dudl);
      }
  };
  exclusion(old_atoms, n_old, 1.0);
  exclusion(new_atoms, n_new, -1.0);
  // self energy (ewald.cpp:1221-1238)
  const double prefactor_self = C * alpha / std::sqrt(rg::kPi);
  for (int i = 0; i < n_old; ++i)
  {
    const double q = old_atoms[i].charge, sc = old_atoms[i].scaling_coulomb;
    const int g = groupOf(old_atoms[i]);
    out->ewald_self += prefactor_self * sc * q * sc * q;
    if (g != 0) out->dudlambda_ewald[g - 1] += 2.0 * prefactor_self * sc * q * q;
  }
  for (int i = 0; i < n_new; ++i)
  {
    const double q = new_atoms[i].charge, sc = new_atoms[i].scaling_coulomb;
    const int g = groupOf(new_atoms[i]);
    out->ewald_self -= prefactor_self * sc * q * sc * q;
    if (g != 0) out->dudlambda_ewald[g - 1] -= 2.0 * prefactor_self * sc * q * q;
  }
  // net-charge correction difference (ewald.cpp:181-208)
  double deltaCharge = 0.0, dNew[4], dOld[4];
  for (int g = 0; g < 4; ++g) dNew[g] = dOld[g] = net_charge_derivative_ext ? net_charge_derivative_ext[g] : 0.0;
  for (int i = 0; i < n_old; ++i)
  {
    deltaCharge -= old_atoms[i].scaling_coulomb * old_atoms[i].charge;
    const int g = groupOf(old_atoms[i]);
    if (g != 0) dOld[g - 1] += old_atoms[i].charge;
  }
  for (int i = 0; i < n_new; ++i)
  {
    deltaCharge += new_atoms[i].scaling_coulomb * new_atoms[i].charge;
    const int g = groupOf(new_atoms[i]);
    if (g != 0) dNew[g - 1] += new_atoms[i].charge;
  }
  const double uIon = -(e->single_ion_sum - C * alpha / std::sqrt(rg::kPi));
  const double netChargeNew = net_charge + deltaCharge;
  out->ewald_fourier += uIon * (netChargeNew * netChargeNew - net_charge * net_charge);
  for (int g = 0; g < 4; ++g) out->dudlambda_ewald[g] += 2.0 * uIon * (netChargeNew * dNew[g] - net_charge * dOld[g]);
  return RG_OK;
}

rg_status rg_ewald_accept(rg_ewald* e)
{
  if (!e) return RG_ERR_INVALID_ARGUMENT;
  if (!e->use_charge) return RG_OK;
  // acceptEwaldMove (ewald.cpp:1565-1574): storedEik = trialEik, done as a pointer swap
  double2* t = e->stored;
  e->stored = e->trial;
  e->trial = t;
  return RG_OK;
}

rg_status rg_ewald_get_structure_factors(rg_ewald* e, int which, double* host, int64_t n_doubles)
{
  if (!e || !host) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  const int64_t need = 2 * e->nk * (1 + e->n_groups);
  if (n_doubles < need) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_get_structure_factors: buffer too small");
  const double2* src = which == 0 ? e->stored : (which == 1 ? e->trial : e->s_rigid);
  const int64_t cnt = which == 2 ? 2 * e->nk : need;
  RG_CUDA(ctx, cudaMemcpyAsync(host, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

rg_status rg_ewald_set_structure_factors(rg_ewald* e, const double* host, int64_t n_doubles)
{
  if (!e || !host) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  const int64_t need = 2 * e->nk * (1 + e->n_groups);
  if (n_doubles != need) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_set_structure_factors: size");
  RG_CUDA(ctx, cudaMemcpyAsync(e->stored, host, sizeof(double) * need, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}
}

namespace rgd
{
rg_status ewaldExport(rg_ewald* e, const char4** kvec, const double** temp, const double2** s_rigid, int64_t* nk,
                      int kmax[3], double* alpha, double* single_ion_sum)
{
  if (!e) return RG_ERR_INVALID_ARGUMENT;
  *kvec = e->kvec;
  *temp = e->temp;
  *s_rigid = e->s_rigid;
  *nk = e->nk;
  kmax[0] = e->ff.kmax_x;
  kmax[1] = e->ff.kmax_y;
  kmax[2] = e->ff.kmax_z;
  *alpha = e->alpha;
  *single_ion_sum = e->single_ion_sum;
  return RG_OK;
}
}  // namespace rgd

// ---------------------------------------------------------------------------------------------------------------------
// The structure-factor update of many systems in one launch (the Fourier part of energyDifferenceEwaldFourier,
// ewald.cpp:1098-1162, for one move in each of n systems that share the box, the force field and the k-vectors).
//
// Each system keeps two structure-factor buffers, stored and trial, and a flag says which is which; an accepted move
// flips its system's flag (acceptEwaldMove, ewald.cpp:1565-1574, without a copy). The launch is (k-tile, system): a
// block loads its system's moved atoms, builds their phase tables e^{i 2 pi m s_d} (m = 0..kmax_d) in shared memory,
// and every thread forms Delta rho(k) of its k-vectors from two complex products per atom, reads S(k), writes
// S(k) + Delta rho(k) and sums temp(k) (2 Re(conj(S) Delta rho) + |Delta rho|^2). Block partials are reduced per system
// in block order by the system's last block, which writes the total into mapped pinned host memory. The traffic per
// system and move is 32 bytes per k-vector (read S, write the trial S); k-vectors and prefactors are shared by all
// systems and stay in L2.
// ---------------------------------------------------------------------------------------------------------------------
struct rg_ewald_batch
{
  rg_ewald* ewald = nullptr;
  int n = 0;
  int max_atoms = 0;
  double2* sk = nullptr;           // [2][n][nk]
  unsigned char* cur = nullptr;    // [n]: which buffer holds the stored S(k) of system s
  std::vector<unsigned char> cur_host;
  MovedAtom* atoms = nullptr;      // [n][kBatchAtoms] device
  MovedAtom* atoms_host = nullptr; // pinned
  int* counts = nullptr;           // [n] moved atoms per system (device)
  int* counts_host = nullptr;      // pinned
  double* partial = nullptr;       // [n][blocks]
  unsigned int* counter = nullptr; // [n]
  double* result = nullptr;        // device view of result_host
  double* result_host = nullptr;   // [n] mapped pinned
  int blocks = 0;                  // k-ranges per system
  int4* desc = nullptr;            // [blocks]: first k, end k, first (kx, ky) pair, pairs
  int* kinfo = nullptr;            // [nk]: pair * 256 + (kz + 128)
  char2* pairs = nullptr;          // [pairs]: (kx, ky)
  // device time of the last rg_ewald_batch_delta: events before the atom upload, before and after the kernel
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  float upload_ms = 0.0f, kernel_ms = 0.0f;
};

namespace
{
constexpr int kBatchAtoms = 16;       // old + new atoms of one system's move
constexpr int kBatchKPerThread = 8;   // k-vectors per thread: a block covers at most kThreads * 8 of them
constexpr int kBatchPairs = 128;      // (kx, ky) pairs of one block's k-range

// Shared memory of a block: the phasor tables exp(2 pi i m s_d) of its system's moved atoms (x: m = 0..kmax_x; y and z:
// m = -kmax..kmax, the negative m as conjugates) and the weighted xy products of its (kx, ky) pairs.
__host__ __device__ inline size_t batchSharedBytes(int stride, int kxm, int kym, int kzm)
{
  return sizeof(double2) * static_cast<size_t>(stride) * ((kxm + 1) + (2 * kym + 1) + (2 * kzm + 1) + kBatchPairs);
}

// One block per (k-range, system). The k-vectors come in the reference's order (kx outer, then ky, then kz), so a
// k-range spans few (kx, ky) pairs: the block forms w_a exp(2 pi i (kx s_a,x + ky s_a,y)) once per pair and atom, and
// each k then costs one complex multiply-add per atom with its z phasor. desc[b] = {first k, end k, first pair,
// pairs}; kinfo[k] = pair * 256 + (kz + 128); pairs[p] = (kx, ky).
__global__ void __launch_bounds__(kThreads) ewaldBatchDeltaKernel(
    const int4* __restrict__ desc, const int* __restrict__ kinfo, const char2* __restrict__ pairs, int64_t nk,
    int n_systems, const double* __restrict__ temp, double2* sk, const unsigned char* __restrict__ cur,
    const MovedAtom* __restrict__ atoms, int atom_stride, const int* __restrict__ counts, int kxm, int kym, int kzm,
    double* partial, unsigned int* counter, double* result)
{
  extern __shared__ double2 tab[];
  __shared__ double red[kThreads / 32];
  __shared__ bool last;
  const int sys = blockIdx.y;
  const int4 d = desc[blockIdx.x];
  const int na = counts[sys];
  const int nx = kxm + 1, ny = 2 * kym + 1, nz = 2 * kzm + 1;
  double2* ex = tab;
  double2* ey = ex + atom_stride * nx;
  double2* ez = ey + atom_stride * ny;
  double2* wxy = ez + atom_stride * nz;  // [pair][atom]
  const MovedAtom* ma = atoms + static_cast<long long>(sys) * atom_stride;
  const int per = nx + (kym + 1) + (kzm + 1);
  for (int idx = threadIdx.x; idx < na * per; idx += blockDim.x)
  {
    const int a = idx / per, m = idx - a * per;
    const int dim = m < nx ? 0 : (m < nx + kym + 1 ? 1 : 2);
    const int mm = dim == 0 ? m : (dim == 1 ? m - nx : m - nx - (kym + 1));
    double sn, cs;
    sincospi(2.0 * static_cast<double>(mm) * ma[a].s[dim], &sn, &cs);
    if (dim == 0)
      ex[a * nx + mm] = make_double2(cs, sn);
    else if (dim == 1)
    {
      ey[a * ny + kym + mm] = make_double2(cs, sn);
      ey[a * ny + kym - mm] = make_double2(cs, -sn);
    }
    else
    {
      ez[a * nz + kzm + mm] = make_double2(cs, sn);
      ez[a * nz + kzm - mm] = make_double2(cs, -sn);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < d.w * na; idx += blockDim.x)
  {
    const int j = idx / na, a = idx - j * na;
    const char2 pq = pairs[d.z + j];
    const double2 x = ex[a * nx + pq.x], y = ey[a * ny + kym + pq.y];
    const double w = ma[a].w;
    wxy[j * atom_stride + a] = make_double2(w * (x.x * y.x - x.y * y.y), w * (x.x * y.y + x.y * y.x));
  }
  __syncthreads();
  const double2* S = sk + (static_cast<long long>(cur[sys]) * n_systems + sys) * nk;
  double2* T = sk + (static_cast<long long>(1 - cur[sys]) * n_systems + sys) * nk;
  double e = 0.0;
#pragma unroll
  for (int r = 0; r < kBatchKPerThread; ++r)
  {
    const int k = d.x + r * kThreads + static_cast<int>(threadIdx.x);
    if (k >= d.y) continue;
    const int info = kinfo[k];
    const double2* w = wxy + ((info >> 8) - d.z) * atom_stride;
    const double2* z = ez + (info & 0xff) - 128 + kzm;
    double2 dr = make_double2(0.0, 0.0);
    for (int a = 0; a < na; ++a)
    {
      const double2 wa = w[a], za = z[a * nz];
      dr.x = fma(wa.x, za.x, fma(-wa.y, za.y, dr.x));
      dr.y = fma(wa.x, za.y, fma(wa.y, za.x, dr.y));
    }
    const double2 s = __ldcs(S + k);
    e += temp[k] * (2.0 * (s.x * dr.x + s.y * dr.y) + (dr.x * dr.x + dr.y * dr.y));
    __stcs(T + k, make_double2(s.x + dr.x, s.y + dr.y));
  }
  // fixed-order reduction: warps, then the block, then (the system's last block) the blocks in order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if (lane == 0) red[warp] = e;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double x = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) x += red[q];
    partial[static_cast<long long>(sys) * gridDim.x + blockIdx.x] = x;
    __threadfence();
    last = atomicAdd(counter + sys, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double y = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
    y += __ldcg(partial + static_cast<long long>(sys) * gridDim.x + b);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) y += __shfl_down_sync(0xffffffffu, y, o);
  if (lane == 0) red[warp] = y;
  __syncthreads();
  if (threadIdx.x == 0)
  {
    double x = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) x += red[q];
    result[sys] = x;
    counter[sys] = 0u;  // ready for the next launch
  }
}
}  // namespace

extern "C"
{
rg_status rg_ewald_batch_create(rg_ewald* e, int n_systems, rg_ewald_batch** out)
{
  if (!e || !out || n_systems < 1 || n_systems > 65535) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = e->ctx;
  if (e->n_groups != 0)
    return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_ewald_batch_create: the batch carries no dU/dlambda groups");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_ewald_batch* b = new rg_ewald_batch();
  b->ewald = e;
  b->n = n_systems;
  const int64_t nk = std::max<int64_t>(1, e->nk);
  // k-ranges of at most kThreads * kBatchKPerThread k-vectors and kBatchPairs (kx, ky) pairs, from the k-vector list
  std::vector<char4> kv(static_cast<size_t>(e->nk));
  std::vector<int> kinfo(static_cast<size_t>(nk), 0);
  std::vector<char2> pairs;
  std::vector<int4> desc;
  cudaError_t err = cudaSuccess;
  if (e->nk > 0)
  {
    err = cudaMemcpyAsync(kv.data(), e->kvec, sizeof(char4) * e->nk, cudaMemcpyDeviceToHost, ctx->stream);
    if (!err) err = cudaStreamSynchronize(ctx->stream);
  }
  if (err)
  {
    delete b;
    return rg::cudaFail(ctx, err, "rg_ewald_batch_create");
  }
  for (int64_t k = 0; k < e->nk; ++k)
  {
    if (k == 0 || kv[k].x != kv[k - 1].x || kv[k].y != kv[k - 1].y) pairs.push_back(make_char2(kv[k].x, kv[k].y));
    kinfo[k] = static_cast<int>(pairs.size() - 1) * 256 + (kv[k].z + 128);
  }
  for (int64_t k0 = 0; k0 < e->nk;)
  {
    const int p0 = kinfo[k0] >> 8;
    int64_t k1 = k0;
    while (k1 < e->nk && k1 - k0 < kThreads * kBatchKPerThread && (kinfo[k1] >> 8) - p0 < kBatchPairs) ++k1;
    desc.push_back(make_int4(static_cast<int>(k0), static_cast<int>(k1), p0, (kinfo[k1 - 1] >> 8) - p0 + 1));
    k0 = k1;
  }
  if (desc.empty()) desc.push_back(make_int4(0, 0, 0, 0));
  if (pairs.empty()) pairs.push_back(make_char2(0, 0));
  b->blocks = static_cast<int>(desc.size());
  err = cudaMalloc(reinterpret_cast<void**>(&b->desc), sizeof(int4) * desc.size());
  if (!err) err = cudaMemcpyAsync(b->desc, desc.data(), sizeof(int4) * desc.size(), cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->kinfo), sizeof(int) * kinfo.size());
  if (!err) err = cudaMemcpyAsync(b->kinfo, kinfo.data(), sizeof(int) * kinfo.size(), cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->pairs), sizeof(char2) * pairs.size());
  if (!err) err = cudaMemcpyAsync(b->pairs, pairs.data(), sizeof(char2) * pairs.size(), cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->sk), sizeof(double2) * 2 * n_systems * nk);
  if (!err) err = cudaMemsetAsync(b->sk, 0, sizeof(double2) * 2 * n_systems * nk, ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->cur), n_systems);
  if (!err) err = cudaMemsetAsync(b->cur, 0, n_systems, ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->atoms), sizeof(MovedAtom) * kBatchAtoms * n_systems);
  if (!err) err = cudaMallocHost(reinterpret_cast<void**>(&b->atoms_host), sizeof(MovedAtom) * kBatchAtoms * n_systems);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->counts), sizeof(int) * n_systems);
  if (!err) err = cudaMallocHost(reinterpret_cast<void**>(&b->counts_host), sizeof(int) * n_systems);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->partial), sizeof(double) * n_systems * b->blocks);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&b->counter), sizeof(unsigned int) * n_systems);
  if (!err) err = cudaMemsetAsync(b->counter, 0, sizeof(unsigned int) * n_systems, ctx->stream);
  if (!err) err = cudaHostAlloc(reinterpret_cast<void**>(&b->result_host), sizeof(double) * n_systems, cudaHostAllocMapped);
  if (!err) err = cudaHostGetDevicePointer(reinterpret_cast<void**>(&b->result), b->result_host, 0);
  for (int i = 0; i < 3 && !err; ++i) err = cudaEventCreate(&b->ev[i]);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (err)
  {
    rg_status st = rg::cudaFail(ctx, err, "rg_ewald_batch_create");
    rg_ewald_batch_destroy(b);
    return st;
  }
  b->cur_host.assign(n_systems, 0);
  *out = b;
  return RG_OK;
}

rg_status rg_ewald_batch_destroy(rg_ewald_batch* b)
{
  if (!b) return RG_OK;
  if (b->ewald && b->ewald->ctx) cudaStreamSynchronize(b->ewald->ctx->stream);
  cudaFree(b->sk);
  cudaFree(b->cur);
  cudaFree(b->atoms);
  cudaFree(b->counts);
  cudaFree(b->partial);
  cudaFree(b->counter);
  cudaFree(b->desc);
  cudaFree(b->kinfo);
  cudaFree(b->pairs);
  if (b->atoms_host) cudaFreeHost(b->atoms_host);
  if (b->counts_host) cudaFreeHost(b->counts_host);
  if (b->result_host) cudaFreeHost(b->result_host);
  for (cudaEvent_t ev : b->ev)
    if (ev) cudaEventDestroy(ev);
  delete b;
  return RG_OK;
}

rg_status rg_ewald_batch_set(rg_ewald_batch* b, int system, const double* sk)
{
  if (!b || system < 0 || system >= b->n) return RG_ERR_INVALID_ARGUMENT;
  rg_ewald* e = b->ewald;
  rg_ctx* ctx = e->ctx;
  if (e->nk == 0) return RG_OK;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  double2* dst = b->sk + (static_cast<long long>(b->cur_host[system]) * b->n + system) * e->nk;
  if (sk)
  {
    for (int64_t i = 0; i < 2 * e->nk; ++i)
      if (!std::isfinite(sk[i])) return rg::fail(ctx, RG_ERR_NONFINITE, "rg_ewald_batch_set: NaN or infinite S(k)");
    RG_CUDA(ctx, cudaMemcpyAsync(dst, sk, sizeof(double2) * e->nk, cudaMemcpyHostToDevice, ctx->stream));
  }
  else  // the Ewald state's stored total structure factor (entry 0 of each k)
    RG_CUDA(ctx, cudaMemcpy2DAsync(dst, sizeof(double2), e->stored, sizeof(double2) * (1 + e->n_groups),
                                   sizeof(double2), e->nk, cudaMemcpyDeviceToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

rg_status rg_ewald_batch_get(rg_ewald_batch* b, int system, int which, double* sk)
{
  if (!b || !sk || system < 0 || system >= b->n || (which != 0 && which != 1)) return RG_ERR_INVALID_ARGUMENT;
  rg_ewald* e = b->ewald;
  rg_ctx* ctx = e->ctx;
  if (e->nk == 0) return RG_OK;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int buf = which == 0 ? b->cur_host[system] : 1 - b->cur_host[system];
  RG_CUDA(ctx, cudaMemcpyAsync(sk, b->sk + (static_cast<long long>(buf) * b->n + system) * e->nk,
                               sizeof(double2) * e->nk, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

rg_status rg_ewald_batch_delta(rg_ewald_batch* b, const rg_atom* atoms, int max_atoms, const int32_t* n_new,
                               const int32_t* n_old, double* delta_fourier)
{
  if (!b || !atoms || !n_new || !n_old || !delta_fourier || max_atoms < 1) return RG_ERR_INVALID_ARGUMENT;
  rg_ewald* e = b->ewald;
  rg_ctx* ctx = e->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  // the staging buffers are free: every call ends by synchronising the stream; system s's atoms are packed at
  // s * stride (stride = max_atoms, at most kBatchAtoms)
  const int stride = std::min(max_atoms, kBatchAtoms);
  for (int s = 0; s < b->n; ++s)
  {
    if (n_new[s] < 0 || n_old[s] < 0 || n_new[s] + n_old[s] > std::min(max_atoms, kBatchAtoms))
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_ewald_batch_delta: at most 16 old + new atoms per system");
    const rg_atom* a = atoms + static_cast<long long>(s) * max_atoms;
    if (rg_status fs = rg::checkFinite(ctx, a, n_new[s] + n_old[s], "rg_ewald_batch_delta")) return fs;
    // new atoms with +q, then old atoms with -q (packMoved takes the old ones first)
    packMoved(e, a + n_new[s], n_old[s], a, n_new[s], -1.0, b->atoms_host + static_cast<long long>(s) * stride);
    b->counts_host[s] = e->use_charge ? n_new[s] + n_old[s] : 0;
  }
  if (e->nk == 0 || !e->use_charge)
  {
    for (int s = 0; s < b->n; ++s) delta_fourier[s] = 0.0;
    return RG_OK;
  }
  RG_CUDA(ctx, cudaEventRecord(b->ev[0], ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(b->atoms, b->atoms_host, sizeof(MovedAtom) * stride * b->n, cudaMemcpyHostToDevice,
                               ctx->stream));
  RG_CUDA(ctx, cudaMemcpyAsync(b->counts, b->counts_host, sizeof(int) * b->n, cudaMemcpyHostToDevice, ctx->stream));
  const int kxm = e->ff.kmax_x, kym = e->ff.kmax_y, kzm = e->ff.kmax_z;
  const size_t shmem = batchSharedBytes(stride, kxm, kym, kzm);
  if (shmem > 200 * 1024)
    return rg::fail(ctx, RG_ERR_UNSUPPORTED, "rg_ewald_batch_delta: kmax too large for the shared-memory tables");
  RG_CUDA(ctx, cudaFuncSetAttribute(ewaldBatchDeltaKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(shmem)));
  dim3 grid(b->blocks, b->n);
  RG_CUDA(ctx, cudaEventRecord(b->ev[1], ctx->stream));
  ewaldBatchDeltaKernel<<<grid, kThreads, shmem, ctx->stream>>>(b->desc, b->kinfo, b->pairs, e->nk, b->n, e->temp,
                                                               b->sk, b->cur, b->atoms, stride, b->counts, kxm, kym,
                                                               kzm, b->partial, b->counter, b->result);
  RG_CUDA(ctx, cudaGetLastError());
  RG_CUDA(ctx, cudaEventRecord(b->ev[2], ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  RG_CUDA(ctx, cudaEventElapsedTime(&b->upload_ms, b->ev[0], b->ev[1]));
  RG_CUDA(ctx, cudaEventElapsedTime(&b->kernel_ms, b->ev[1], b->ev[2]));
  std::memcpy(delta_fourier, b->result_host, sizeof(double) * b->n);
  return RG_OK;
}

rg_status rg_ewald_batch_timing(rg_ewald_batch* b, float* upload_ms, float* kernel_ms)
{
  if (!b) return RG_ERR_INVALID_ARGUMENT;
  if (upload_ms) *upload_ms = b->upload_ms;
  if (kernel_ms) *kernel_ms = b->kernel_ms;
  return RG_OK;
}

rg_status rg_ewald_batch_accept(rg_ewald_batch* b, const uint8_t* accept)
{
  if (!b || !accept) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = b->ewald->ctx;
  bool any = false;
  for (int s = 0; s < b->n; ++s)
    if (accept[s])
    {
      b->cur_host[s] ^= 1;
      any = true;
    }
  if (!any) return RG_OK;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  RG_CUDA(ctx, cudaMemcpyAsync(b->cur, b->cur_host.data(), b->n, cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}
}  // extern "C"

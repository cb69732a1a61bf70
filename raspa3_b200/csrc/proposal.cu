// Learned first-bead insertion proposal: a Fourier-feature MLP trained on grid Boltzmann factors, tabulated into an
// exactly normalised, exactly samplable density.
//
// There is no counterpart in RASPA3; the proposal replaces the uniform first-bead positions of
// CBMC::growMoleculeMultipleFirstBeadSwapInsertion (src/raspakit/cbmc/multiple_first_bead.cpp:23-27) and the k-1 new
// positions of retraceMultipleFirstBeadSwapDeletion (:56-61). With trial positions drawn from a density q (per unit
// volume, relative to uniform), the Rosenbluth weight of trial i becomes exp(-beta U_i) / q(r_i); W = sum / k is then
// used in the unchanged insertion / deletion acceptance rules, which keeps detailed balance (biased-CBMC identity).
//
// Network: features phi(s) = {sin, cos}(2 pi n s_a), n = 1..16, a = x, y, z (96 inputs) of the fractional position in
// the framework unit cell; two hidden layers of 64 with SiLU; one output f(s), an unnormalised log-density. Training
// minimises (1/B) sum (f(s_i) - t_i)^2 with Adam, where t_i = max(-beta U(s_i), t_min) and U is the first bead's
// framework energy from the tricubic grids (VDW grid + q times the unit-charge Ewald grid) at uniform random s_i.
//
// Kernels (all FP32, hand-written, no tensor cores: the layers are 64-wide): a CTA takes a tile of 64 samples, keeps
// the weights and the tile's activations in shared memory and runs the layer products as shared-memory tile loops;
// the backward pass writes each CTA's gradient partial, and one more kernel sums the partials in a fixed order and
// applies Adam. Tabulation: f at the centres of G^3 cells of the unit cell; cell probabilities p_c ~ exp(f_c), mixed
// with a uniform density: q(s) = (1 - eps) G^3 p_c(s) + eps. Sampling: with probability eps a uniform position,
// else a cell by binary search of the cumulative p_c and a uniform position inside it.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"

namespace
{
constexpr int kIn = 96, kH = 64;
constexpr int kParams = kH * kIn + kH + kH * kH + kH + kH + 1;  // 10433
constexpr int kOffW1 = 0, kOffB1 = kH * kIn, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH,
              kOffB3 = kOffW3 + kH;
constexpr int kTile = 32;  // samples per CTA: a batch of 4,096 spreads over 128 CTAs (one per SM)
constexpr int kThreads = 256;
constexpr int kLdIn = kIn + 1, kLdH = kH + 1;  // padded leading dimensions (no shared-memory bank conflicts)

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z)
{
  const float sg = 1.0f / (1.0f + __expf(-z));
  return sg * (1.0f + z * (1.0f - sg));
}

struct MlpShared
{
  float W1[kH * kLdIn];
  float W2[kH * kLdH];
  float b1[kH], b2[kH], w3[kH];
  float b3;
  float phi[kTile * kLdIn];
  float z1[kTile * kLdH];
  float h1[kTile * kLdH];
  float z2[kTile * kLdH];
  float h2[kTile * kLdH];
  float f[kTile];
  float df[kTile];
  float lossPart[kThreads / 32];
};

__device__ void loadWeights(MlpShared& S, const float* theta)
{
  for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x) S.W1[(i / kIn) * kLdIn + (i % kIn)] = theta[kOffW1 + i];
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) S.W2[(i / kH) * kLdH + (i % kH)] = theta[kOffW2 + i];
  for (int i = threadIdx.x; i < kH; i += blockDim.x)
  {
    S.b1[i] = theta[kOffB1 + i];
    S.b2[i] = theta[kOffB2 + i];
    S.w3[i] = theta[kOffW3 + i];
  }
  if (threadIdx.x == 0) S.b3 = theta[kOffB3];
}

// phi rows for the tile's samples (fractional positions s[3 * idx])
__device__ void features(MlpShared& S, const float* s, const int* idx, int count)
{
  for (int q = threadIdx.x; q < kTile * 48; q += blockDim.x)
  {
    const int i = q / 48, r = q % 48, a = r / 16, n = r % 16 + 1;
    float sn = 0.0f, cs = 0.0f;
    if (i < count) sincospif(2.0f * static_cast<float>(n) * s[3 * idx[i] + a], &sn, &cs);
    S.phi[i * kLdIn + 32 * a + 2 * (n - 1)] = sn;
    S.phi[i * kLdIn + 32 * a + 2 * (n - 1) + 1] = cs;
  }
}

__device__ void forward(MlpShared& S)
{
  __syncthreads();
  for (int q = threadIdx.x; q < kTile * kH; q += blockDim.x)
  {
    const int i = q / kH, j = q % kH;
    float acc = S.b1[j];
#pragma unroll 8
    for (int k = 0; k < kIn; ++k) acc += S.phi[i * kLdIn + k] * S.W1[j * kLdIn + k];
    S.z1[i * kLdH + j] = acc;
    S.h1[i * kLdH + j] = silu(acc);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kTile * kH; q += blockDim.x)
  {
    const int i = q / kH, j = q % kH;
    float acc = S.b2[j];
#pragma unroll 8
    for (int k = 0; k < kH; ++k) acc += S.h1[i * kLdH + k] * S.W2[j * kLdH + k];
    S.z2[i * kLdH + j] = acc;
    S.h2[i * kLdH + j] = silu(acc);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTile; i += blockDim.x)
  {
    float acc = S.b3;
    for (int k = 0; k < kH; ++k) acc += S.h2[i * kLdH + k] * S.w3[k];
    S.f[i] = acc;
  }
  __syncthreads();
}

// One tile's loss and gradient partial. Samples: idx[] into s/target; batch size B scales the loss.
__global__ void __launch_bounds__(kThreads) mlpGradKernel(const float* __restrict__ theta, const float* __restrict__ s,
                                                          const float* __restrict__ target, int64_t n_samples,
                                                          const int64_t* __restrict__ indices, int batch,
                                                          unsigned long long seed, long long step,
                                                          float* __restrict__ partial, float* __restrict__ lossPartial)
{
  extern __shared__ unsigned char smraw[];
  MlpShared& S = *reinterpret_cast<MlpShared*>(smraw);
  __shared__ int idx[kTile];
  const int tile0 = blockIdx.x * kTile;
  const int count = min(kTile, batch - tile0);
  for (int i = threadIdx.x; i < kTile; i += blockDim.x)
  {
    int64_t k = 0;
    if (i < count)
    {
      if (indices)
        k = indices[tile0 + i];
      else
      {
        // random sample of this training step (splitmix64 of seed, step, slot)
        unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * static_cast<unsigned long long>(step * batch + tile0 + i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        k = static_cast<int64_t>(z % static_cast<unsigned long long>(n_samples));
      }
    }
    idx[i] = static_cast<int>(k);
  }
  loadWeights(S, theta);
  __syncthreads();
  features(S, s, idx, count);
  forward(S);
  // dL/df = 2 (f - t) / B ; loss partial
  float lp = 0.0f;
  for (int i = threadIdx.x; i < kTile; i += blockDim.x)
  {
    float d = 0.0f;
    if (i < count)
    {
      const float r = S.f[i] - target[idx[i]];
      d = 2.0f * r / static_cast<float>(batch);
      lp += r * r;
    }
    S.df[i] = d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lp += __shfl_down_sync(0xffffffffu, lp, o);
  if ((threadIdx.x & 31) == 0) S.lossPart[threadIdx.x >> 5] = lp;
  __syncthreads();
  float* g = partial + static_cast<long long>(blockIdx.x) * kParams;
  // w3, b3 gradients; dz2 = df * w3 * silu'(z2) overwrites z2
  for (int j = threadIdx.x; j < kH; j += blockDim.x)
  {
    float acc = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.df[i] * S.h2[i * kLdH + j];
    g[kOffW3 + j] = acc;
  }
  if (threadIdx.x == 0)
  {
    float acc = 0.0f, l = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.df[i];
    g[kOffB3] = acc;
    for (int w = 0; w < kThreads / 32; ++w) l += S.lossPart[w];
    lossPartial[blockIdx.x] = l;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kTile * kH; q += blockDim.x)
  {
    const int i = q / kH, j = q % kH;
    S.z2[i * kLdH + j] = S.df[i] * S.w3[j] * dsilu(S.z2[i * kLdH + j]);
  }
  __syncthreads();
  // W2, b2 gradients: dz2^T h1
  for (int q = threadIdx.x; q < kH * kH; q += blockDim.x)
  {
    const int j = q / kH, k = q % kH;
    float acc = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.z2[i * kLdH + j] * S.h1[i * kLdH + k];
    g[kOffW2 + q] = acc;
  }
  for (int j = threadIdx.x; j < kH; j += blockDim.x)
  {
    float acc = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.z2[i * kLdH + j];
    g[kOffB2 + j] = acc;
  }
  // dz1 = (dz2 W2) * silu'(z1), into h2 (free now)
  for (int q = threadIdx.x; q < kTile * kH; q += blockDim.x)
  {
    const int i = q / kH, k = q % kH;
    float acc = 0.0f;
#pragma unroll 8
    for (int j = 0; j < kH; ++j) acc += S.z2[i * kLdH + j] * S.W2[j * kLdH + k];
    S.h2[i * kLdH + k] = acc * dsilu(S.z1[i * kLdH + k]);
  }
  __syncthreads();
  // W1, b1 gradients: dz1^T phi
  for (int q = threadIdx.x; q < kH * kIn; q += blockDim.x)
  {
    const int j = q / kIn, k = q % kIn;
    float acc = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.h2[i * kLdH + j] * S.phi[i * kLdIn + k];
    g[kOffW1 + q] = acc;
  }
  for (int j = threadIdx.x; j < kH; j += blockDim.x)
  {
    float acc = 0.0f;
    for (int i = 0; i < kTile; ++i) acc += S.h2[i * kLdH + j];
    g[kOffB1 + j] = acc;
  }
}

// Sum of the tile partials in tile order; with lr > 0 also an Adam step (Kingma & Ba 2015).
__global__ void reduceAdamKernel(float* __restrict__ theta, float* __restrict__ m, float* __restrict__ v,
                                 const float* __restrict__ partial, int n_tiles, float lr, float b1, float b2,
                                 float eps, long long t, float* __restrict__ grad_out,
                                 const float* __restrict__ lossPartial, float* __restrict__ loss_out, int batch)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && loss_out)
  {
    float l = 0.0f;
    for (int b = 0; b < n_tiles; ++b) l += lossPartial[b];
    *loss_out = l / static_cast<float>(batch);
  }
  if (p >= kParams) return;
  float gsum = 0.0f;
  for (int b = 0; b < n_tiles; ++b) gsum += partial[static_cast<long long>(b) * kParams + p];
  if (grad_out) grad_out[p] = gsum;
  if (lr > 0.0f)
  {
    const float mm = b1 * m[p] + (1.0f - b1) * gsum;
    const float vv = b2 * v[p] + (1.0f - b2) * gsum * gsum;
    m[p] = mm;
    v[p] = vv;
    const float mh = mm / (1.0f - powf(b1, static_cast<float>(t)));
    const float vh = vv / (1.0f - powf(b2, static_cast<float>(t)));
    theta[p] -= lr * mh / (sqrtf(vh) + eps);
  }
}

__global__ void __launch_bounds__(kThreads) mlpForwardKernel(const float* __restrict__ theta,
                                                             const float* __restrict__ s, int64_t n,
                                                             float* __restrict__ out)
{
  extern __shared__ unsigned char smraw[];
  MlpShared& S = *reinterpret_cast<MlpShared*>(smraw);
  __shared__ int idx[kTile];
  const long long tile0 = static_cast<long long>(blockIdx.x) * kTile;
  const int count = static_cast<int>(min(static_cast<long long>(kTile), n - tile0));
  for (int i = threadIdx.x; i < kTile; i += blockDim.x) idx[i] = static_cast<int>(i < count ? tile0 + i : tile0);
  loadWeights(S, theta);
  __syncthreads();
  features(S, s, idx, count);
  forward(S);
  for (int i = threadIdx.x; i < count; i += blockDim.x) out[tile0 + i] = S.f[i];
}

// Grid-sampled Boltzmann targets of one bead: s uniform in the unit cell, t = max(-beta U(s), t_min) with
// U = VDW grid + q * unit-charge Ewald grid (the grid branch of cbmc/interactions_framework_molecule.cpp:57-69).
__global__ void sampleTargetsKernel(rgd::Grid vdw, const double* ewald_grid, int quintic, double charge, double beta,
                                    double t_min, double c00, double c01, double c02, double c10, double c11, double c12,
                                    double c20, double c21, double c22, int64_t n, unsigned long long seed,
                                    float* s_out, float* t_out)
{
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u[3];
  for (int a = 0; a < 3; ++a)
  {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * static_cast<unsigned long long>(3 * i + a + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    u[a] = static_cast<double>(z >> 11) * 0x1.0p-53;
  }
  // position = cell * s (columns of the cell are the lattice vectors)
  const double x = c00 * u[0] + c10 * u[1] + c20 * u[2];
  const double y = c01 * u[0] + c11 * u[1] + c21 * u[2];
  const double z = c02 * u[0] + c12 * u[1] + c22 * u[2];
  // the scheme of the system's grids: tricubic (8 values per point) or triquintic (27)
  double e = quintic ? rgd::interpolateQuintic(vdw, x, y, z, nullptr) : rgd::interpolate(vdw, x, y, z);
  if (ewald_grid)
  {
    rgd::Grid ge = vdw;
    ge.data = ewald_grid;
    e += charge * (quintic ? rgd::interpolateQuintic(ge, x, y, z, nullptr) : rgd::interpolate(ge, x, y, z));
  }
  const double t = fmax(-beta * e, t_min);
  s_out[3 * i] = static_cast<float>(u[0]);
  s_out[3 * i + 1] = static_cast<float>(u[1]);
  s_out[3 * i + 2] = static_cast<float>(u[2]);
  t_out[i] = static_cast<float>(t);
}
}  // namespace

struct rg_mlp
{
  rg_ctx* ctx = nullptr;
  float* theta = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* partial = nullptr;
  int partial_tiles = 0;
  float* lossPartial = nullptr;
  float* scalars = nullptr;  // [0] loss
  long long t = 0;           // Adam step count
};

struct rg_proposal
{
  rg_ctx* ctx = nullptr;
  int G = 0;
  double eps = 0.0;
  double* cdf = nullptr;      // inclusive cumulative cell probabilities, G^3
  double* density = nullptr;  // q per cell relative to uniform: (1 - eps) G^3 p_c + eps
  std::vector<double> host_density;
};

namespace rgd
{
rg_status proposalExport(rg_proposal* p, const double** cdf, const double** density, int* G, double* eps)
{
  if (!p) return RG_ERR_INVALID_ARGUMENT;
  *cdf = p->cdf;
  *density = p->density;
  *G = p->G;
  *eps = p->eps;
  return RG_OK;
}
}  // namespace rgd

namespace
{
size_t mlpShared() { return sizeof(MlpShared); }

rg_status ensurePartial(rg_mlp* m, int tiles)
{
  rg_ctx* ctx = m->ctx;
  if (m->partial_tiles >= tiles) return RG_OK;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(m->partial);
  cudaFree(m->lossPartial);
  m->partial = nullptr;
  m->lossPartial = nullptr;
  RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&m->partial), sizeof(float) * kParams * tiles));
  RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&m->lossPartial), sizeof(float) * tiles));
  m->partial_tiles = tiles;
  return RG_OK;
}

rg_status launchGrad(rg_mlp* m, const float* s, const float* t, int64_t n, const int64_t* indices, int batch,
                     unsigned long long seed, long long step)
{
  rg_ctx* ctx = m->ctx;
  const int tiles = (batch + kTile - 1) / kTile;
  rg_status st = ensurePartial(m, tiles);
  if (st) return st;
  const size_t sh = mlpShared();
  cudaFuncSetAttribute(mlpGradKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sh));
  mlpGradKernel<<<tiles, kThreads, sh, ctx->stream>>>(m->theta, s, t, n, indices, batch, seed, step, m->partial,
                                                      m->lossPartial);
  RG_CUDA(ctx, cudaGetLastError());
  return RG_OK;
}
}  // namespace

extern "C"
{
rg_status rg_mlp_create(rg_ctx* ctx, uint64_t seed, rg_mlp** out)
{
  if (!ctx || !out) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  rg_mlp* m = new rg_mlp();
  m->ctx = ctx;
  // He-uniform initial weights (bound sqrt(6 / fan_in)), zero biases, from a seeded splitmix64 stream
  std::vector<float> h(kParams, 0.0f);
  unsigned long long state = seed;
  auto next = [&]()
  {
    state += 0x9E3779B97F4A7C15ULL;
    unsigned long long z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return static_cast<double>(z >> 11) * 0x1.0p-53;
  };
  const double a1 = std::sqrt(6.0 / kIn), a2 = std::sqrt(6.0 / kH);
  for (int i = 0; i < kH * kIn; ++i) h[kOffW1 + i] = static_cast<float>((2.0 * next() - 1.0) * a1);
  for (int i = 0; i < kH * kH; ++i) h[kOffW2 + i] = static_cast<float>((2.0 * next() - 1.0) * a2);
  for (int i = 0; i < kH; ++i) h[kOffW3 + i] = static_cast<float>((2.0 * next() - 1.0) * a2);
  cudaError_t err = cudaMalloc(reinterpret_cast<void**>(&m->theta), sizeof(float) * kParams);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&m->m), sizeof(float) * kParams);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&m->v), sizeof(float) * kParams);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&m->scalars), sizeof(float) * 4);
  // every copy and fill on the context stream: the legacy default stream does not order with it
  if (!err) err = cudaMemcpyAsync(m->theta, h.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMemsetAsync(m->m, 0, sizeof(float) * kParams, ctx->stream);
  if (!err) err = cudaMemsetAsync(m->v, 0, sizeof(float) * kParams, ctx->stream);
  if (!err) err = cudaMemsetAsync(m->scalars, 0, sizeof(float) * 4, ctx->stream);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (err)
  {
    rg_status st = rg::cudaFail(ctx, err, "rg_mlp_create");
    rg_mlp_destroy(m);
    return st;
  }
  *out = m;
  return RG_OK;
}

rg_status rg_mlp_destroy(rg_mlp* m)
{
  if (!m) return RG_OK;
  if (m->ctx) cudaStreamSynchronize(m->ctx->stream);
  cudaFree(m->theta);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->partial);
  cudaFree(m->lossPartial);
  cudaFree(m->scalars);
  delete m;
  return RG_OK;
}

int32_t rg_mlp_num_params(void) { return kParams; }

rg_status rg_mlp_get_params(rg_mlp* m, float* host, int32_t n)
{
  if (!m || !host || n != kParams) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(m->ctx, cudaMemcpyAsync(host, m->theta, sizeof(float) * kParams, cudaMemcpyDeviceToHost, m->ctx->stream));
  RG_CUDA(m->ctx, cudaStreamSynchronize(m->ctx->stream));
  return RG_OK;
}

rg_status rg_mlp_set_params(rg_mlp* m, const float* host, int32_t n)
{
  if (!m || !host || n != kParams) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(m->ctx, cudaMemcpyAsync(m->theta, host, sizeof(float) * kParams, cudaMemcpyHostToDevice, m->ctx->stream));
  RG_CUDA(m->ctx, cudaStreamSynchronize(m->ctx->stream));
  return RG_OK;
}

rg_status rg_mlp_loss_and_gradient(rg_mlp* m, const float* s_device, const float* target_device, int32_t n,
                                   float* loss, float* grad_host)
{
  if (!m || !s_device || !target_device || n < 1 || n > (1 << 24)) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = m->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<int64_t> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  int64_t* didx = nullptr;
  RG_CUDA(ctx, cudaMalloc(reinterpret_cast<void**>(&didx), sizeof(int64_t) * n));
  rg_status st = RG_OK;
  float* dgrad = nullptr;
  cudaError_t err = cudaMemcpyAsync(didx, idx.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&dgrad), sizeof(float) * kParams);
  if (err) st = rg::cudaFail(ctx, err, "rg_mlp_loss_and_gradient");
  if (!st) st = launchGrad(m, s_device, target_device, n, didx, n, 0, 0);
  if (!st)
  {
    const int tiles = (n + kTile - 1) / kTile;
    reduceAdamKernel<<<(kParams + 255) / 256, 256, 0, ctx->stream>>>(m->theta, m->m, m->v, m->partial, tiles, 0.0f,
                                                                     0.f, 0.f, 0.f, 1, dgrad, m->lossPartial,
                                                                     m->scalars, n);
    err = cudaGetLastError();
    if (!err && grad_host)
      err = cudaMemcpyAsync(grad_host, dgrad, sizeof(float) * kParams, cudaMemcpyDeviceToHost, ctx->stream);
    if (!err && loss) err = cudaMemcpyAsync(loss, m->scalars, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (!err) err = cudaStreamSynchronize(ctx->stream);
    if (err) st = rg::cudaFail(ctx, err, "rg_mlp_loss_and_gradient");
  }
  cudaStreamSynchronize(ctx->stream);
  cudaFree(didx);
  cudaFree(dgrad);
  return st;
}

rg_status rg_mlp_train(rg_mlp* m, const float* s_device, const float* target_device, int64_t n_samples, int32_t steps,
                       int32_t batch, float learning_rate, uint64_t seed, float* final_loss)
{
  if (!m || !s_device || !target_device || n_samples < 1 || steps < 0 || batch < 1) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = m->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int tiles = (batch + kTile - 1) / kTile;
  for (int s = 0; s < steps; ++s)
  {
    rg_status st = launchGrad(m, s_device, target_device, n_samples, nullptr, batch, seed, m->t);
    if (st) return st;
    ++m->t;
    reduceAdamKernel<<<(kParams + 255) / 256, 256, 0, ctx->stream>>>(m->theta, m->m, m->v, m->partial, tiles,
                                                                     learning_rate, 0.9f, 0.999f, 1e-8f, m->t, nullptr,
                                                                     m->lossPartial, m->scalars, batch);
    RG_CUDA(ctx, cudaGetLastError());
  }
  if (final_loss)
  {
    RG_CUDA(ctx, cudaMemcpyAsync(final_loss, m->scalars, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  }
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

rg_status rg_mlp_evaluate(rg_mlp* m, const float* s_device, int64_t n, float* out_device)
{
  if (!m || !s_device || !out_device || n < 0) return RG_ERR_INVALID_ARGUMENT;
  if (n == 0) return RG_OK;
  rg_ctx* ctx = m->ctx;
  const size_t sh = mlpShared();
  cudaFuncSetAttribute(mlpForwardKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sh));
  const long long tiles = (n + kTile - 1) / kTile;
  mlpForwardKernel<<<static_cast<unsigned>(tiles), kThreads, sh, ctx->stream>>>(m->theta, s_device, n, out_device);
  RG_CUDA(ctx, cudaGetLastError());
  return RG_OK;
}

rg_status rg_proposal_sample_targets(rg_system* system, int pseudo_atom, double charge, double beta, double t_min,
                                     const rg_box* unit_cell, int64_t n, uint64_t seed, float* s_device,
                                     float* t_device)
{
  if (!system || !unit_cell || n < 1 || !s_device || !t_device) return RG_ERR_INVALID_ARGUMENT;
  rgd::FF ff;
  rgd::Box box;
  const double* grids[64];
  const double* ewald_grid;
  int n_types, gd[3];
  double gic[3][3];
  rg_ctx* ctx;
  rg_status st = rgd::systemExport(system, &ff, &box, grids, &ewald_grid, &n_types, gd, gic, &ctx);
  if (st) return st;
  if (pseudo_atom < 0 || pseudo_atom >= 64 || pseudo_atom >= n_types || !grids[pseudo_atom])
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_proposal_sample_targets: no grid for this pseudo-atom");
  rgd::Grid g{grids[pseudo_atom], gd[0], gd[1], gd[2], {}};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) g.ic[a][b] = gic[a][b];
  const double* c = unit_cell->cell;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  sampleTargetsKernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(
      g, ff.use_charge ? ewald_grid : nullptr, rgd::systemScheme(system) == RG_SCHEME_TRIQUINTIC ? 1 : 0, charge, beta,
      t_min, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], n, seed, s_device, t_device);
  RG_CUDA(ctx, cudaGetLastError());
  return RG_OK;
}

rg_status rg_proposal_create(rg_mlp* m, int32_t cells_per_axis, double eps_uniform, rg_proposal** out)
{
  if (!m || !out || cells_per_axis < 1 || cells_per_axis > 256 || !(eps_uniform > 0.0) || eps_uniform > 1.0)
    return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = m->ctx;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int G = cells_per_axis;
  const int64_t nc = static_cast<int64_t>(G) * G * G;
  std::vector<float> s(3 * nc);
  for (int64_t c = 0; c < nc; ++c)
  {
    const int64_t i = c % G, j = (c / G) % G, k = c / (static_cast<int64_t>(G) * G);
    s[3 * c] = static_cast<float>((i + 0.5) / G);
    s[3 * c + 1] = static_cast<float>((j + 0.5) / G);
    s[3 * c + 2] = static_cast<float>((k + 0.5) / G);
  }
  // cell centres and MLP outputs in the context's scratch slot 6 (no allocation or free per table)
  void* scr = nullptr;
  rg_status st = rg::scratch(ctx, 6, sizeof(float) * 4 * static_cast<size_t>(nc), &scr);
  if (st) return st;
  float* ds = static_cast<float*>(scr);
  float* df = ds + 3 * nc;
  cudaError_t err = cudaMemcpyAsync(ds, s.data(), sizeof(float) * 3 * nc, cudaMemcpyHostToDevice, ctx->stream);
  st = err ? rg::cudaFail(ctx, err, "rg_proposal_create") : rg_mlp_evaluate(m, ds, nc, df);
  std::vector<float> f(nc);
  if (!st)
  {
    err = cudaMemcpyAsync(f.data(), df, sizeof(float) * nc, cudaMemcpyDeviceToHost, ctx->stream);
    if (!err) err = cudaStreamSynchronize(ctx->stream);
    if (err) st = rg::cudaFail(ctx, err, "rg_proposal_create");
  }
  if (st) return st;
  // p_c ~ exp(f_c - max f), cumulative in FP64
  double fmax = -1e300;
  for (float v : f) fmax = std::fmax(fmax, static_cast<double>(v));
  std::vector<double> w(nc), cdf(nc), dens(nc);
  double sum = 0.0;
  for (int64_t c = 0; c < nc; ++c)
  {
    w[c] = std::exp(static_cast<double>(f[c]) - fmax);
    sum += w[c];
  }
  double acc = 0.0;
  for (int64_t c = 0; c < nc; ++c)
  {
    acc += w[c] / sum;
    cdf[c] = acc;
    dens[c] = (1.0 - eps_uniform) * static_cast<double>(nc) * (w[c] / sum) + eps_uniform;
  }
  cdf[nc - 1] = 1.0;
  rg_proposal* p = new rg_proposal();
  p->ctx = ctx;
  p->G = G;
  p->eps = eps_uniform;
  err = cudaMalloc(reinterpret_cast<void**>(&p->cdf), sizeof(double) * nc);
  if (!err) err = cudaMalloc(reinterpret_cast<void**>(&p->density), sizeof(double) * nc);
  if (!err) err = cudaMemcpyAsync(p->cdf, cdf.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaMemcpyAsync(p->density, dens.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, ctx->stream);
  if (!err) err = cudaStreamSynchronize(ctx->stream);
  if (err)
  {
    st = rg::cudaFail(ctx, err, "rg_proposal_create");
    rg_proposal_destroy(p);
    return st;
  }
  p->host_density = dens;
  *out = p;
  return RG_OK;
}

rg_status rg_proposal_destroy(rg_proposal* p)
{
  if (!p) return RG_OK;
  if (p->ctx) cudaStreamSynchronize(p->ctx->stream);
  cudaFree(p->cdf);
  cudaFree(p->density);
  delete p;
  return RG_OK;
}

rg_status rg_proposal_density(rg_proposal* p, const double* s, int64_t n, double* q_out)
{
  if (!p || (n > 0 && (!s || !q_out))) return RG_ERR_INVALID_ARGUMENT;
  const int G = p->G;
  for (int64_t i = 0; i < n; ++i)
  {
    int64_t c[3];
    for (int a = 0; a < 3; ++a)
    {
      double f = s[3 * i + a] - std::floor(s[3 * i + a]);
      c[a] = std::min<int64_t>(G - 1, static_cast<int64_t>(f * G));
    }
    q_out[i] = p->host_density[c[0] + G * (c[1] + static_cast<int64_t>(G) * c[2])];
  }
  return RG_OK;
}
}

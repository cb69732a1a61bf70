// FP32 / FP64 FMA-throughput probe: the SIMT-pipe denominator of the rooflines of the pair kernels (the driver's peak
// table holds only the HBM copy bandwidth and the dense bf16 tensor throughput).
#include "common.cuh"

namespace
{
template <typename T>
__global__ void __launch_bounds__(256) fmaChains(T* out, int iters, T a, T b)
{
  // 8 independent FMA chains per thread keep the pipe busy without depending on memory.
  T x0 = threadIdx.x * T(1e-7), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
  T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
  for (int i = 0; i < iters; ++i)
  {
#pragma unroll
    for (int u = 0; u < 16; ++u)
    {
      x0 = x0 * a + b;
      x1 = x1 * a + b;
      x2 = x2 * a + b;
      x3 = x3 * a + b;
      x4 = x4 * a + b;
      x5 = x5 * a + b;
      x6 = x6 * a + b;
      x7 = x7 * a + b;
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345)) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains alive
}
}  // namespace

extern "C" rg_status rg_probe_fma_peak(rg_ctx* ctx, int precision, double* tflops, double* seconds)
{
  if (!ctx || !tflops) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  int sms = 0;
  RG_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
  const int blocks = sms * 8, threads = 256;
  const int iters = precision == RG_PRECISION_FP64 ? 2048 : 4096;
  void* p = nullptr;
  rg_status st = rg::scratch(ctx, 7, sizeof(double) * blocks * threads, &p);
  if (st) return st;
  cudaEvent_t e0, e1;
  RG_CUDA(ctx, cudaEventCreate(&e0));
  RG_CUDA(ctx, cudaEventCreate(&e1));
  float best_ms = 1e30f;
  for (int rep = 0; rep < 4; ++rep)
  {
    RG_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
    if (precision == RG_PRECISION_FP64)
      fmaChains<double><<<blocks, threads, 0, ctx->stream>>>(static_cast<double*>(p), iters, 0.999999, 1e-9);
    else
      fmaChains<float><<<blocks, threads, 0, ctx->stream>>>(static_cast<float*>(p), iters, 0.999999f, 1e-9f);
    RG_CUDA(ctx, cudaGetLastError());
    RG_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
    RG_CUDA(ctx, cudaEventSynchronize(e1));
    float ms = 0;
    RG_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && ms < best_ms) best_ms = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double flops = 2.0 * 8.0 * 16.0 * iters * static_cast<double>(blocks) * threads;
  *tflops = flops / (best_ms * 1e-3) / 1e12;
  if (seconds) *seconds = best_ms * 1e-3;
  return RG_OK;
}

// Shared host/device helpers of libraspagpu: the context, error plumbing, device scratch and small math.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/raspa_gpu.h"

struct rg_ctx
{
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // Grow-only device scratch slots, reused across calls on this context.
  struct Slot
  {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  std::vector<Slot> scratch;
  // Pinned host staging slots.
  std::vector<Slot> pinned;
  // Second stream for device-to-host copies that overlap the work of `stream`, and events to order the two (created
  // on first use).
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> events;
};

namespace rg
{
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kInvSqrtPi = 0.564189583547756286948079451560772586;

// Unit constants with the reference's expressions (src/raspakit/units.cpp:14-98).
inline double energyConversionFactor() { return 1.6605402e-27 * 1e-10 * 1e-10 / (1e-12 * 1e-12); }
inline double coulombFactor()
{
  return 1.60217733e-19 * 1.60217733e-19 / (4.0 * kPi * 8.8541878176e-12 * 1e-10 * energyConversionFactor());
}

rg_status fail(rg_ctx* ctx, rg_status code, const std::string& msg);
rg_status cudaFail(rg_ctx* ctx, cudaError_t err, const char* what);
// Device scratch slot `slot` of at least `bytes` (grows; contents undefined).
rg_status scratch(rg_ctx* ctx, int slot, size_t bytes, void** out);
// Pinned host slot `slot` of at least `bytes`.
rg_status pinnedScratch(rg_ctx* ctx, int slot, size_t bytes, void** out);
// The context's copy stream and its event `i` (created on first use).
rg_status copyStream(rg_ctx* ctx, cudaStream_t* out);
rg_status event(rg_ctx* ctx, int i, cudaEvent_t* out);
// Makes the context stream wait for everything queued on the copy stream so far.
rg_status joinCopies(rg_ctx* ctx);

// RG_ERR_NONFINITE (with a message naming `what`) if any position, charge or scaling factor of the atoms is NaN or
// infinite, RG_OK otherwise. Host inputs are checked before anything is launched.
rg_status checkFinite(rg_ctx* ctx, const rg_atom* atoms, long long n, const char* what);
rg_status checkFiniteBox(rg_ctx* ctx, const rg_box* box, const char* what);

struct HostBox
{
  double c[3][3];   // c[col][row]
  double ic[3][3];  // inverse, same convention
  bool triclinic;
  double volume;
};
HostBox makeHostBox(const rg_box* b);
void perpendicularWidths(const HostBox& b, double w[3]);
// The supercell that `cutoff` sizes in the reference's grid builds (ceil(2 cutoff / width) unit cells per axis,
// SimulationBox::smallestNumberOfUnitCellsForMinimumImagesConvention, simulationbox.cpp:150-156): half its lengths
// (h, rectangular) and its inverse as ic[d][k] (fraction d from Cartesian k). Returns whether its minimum image can
// drop pairs within the pair cutoff `rc`, i.e. whether it is narrower than 2 rc along some axis.
bool supercellClip(const HostBox& b, double rc, double cutoff, double h[3], double ic[3][3]);
inline void matvec(const double m[3][3], const double v[3], double out[3])
{
  for (int r = 0; r < 3; ++r) out[r] = m[0][r] * v[0] + m[1][r] * v[1] + m[2][r] * v[2];
}
}  // namespace rg

#define RG_CUDA(ctx, call)                                   \
  do                                                         \
  {                                                          \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return rg::cudaFail(ctx, _e, #call); \
  } while (0)

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of 32, <= 1024). `warp_sums` is shared
// scratch of 33 ints; callers separate two scans with a __syncthreads. Returns the exclusive prefix; *total receives the block sum. Contains two __syncthreads.
__device__ __forceinline__ int blockExclusiveScan(int v, int* warp_sums, int* total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0)
  {
    int w = (lane < nwarps) ? warp_sums[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1)
    {
      int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < nwarps) warp_sums[lane] = wi - w;  // exclusive warp offsets
    if (lane == nwarps - 1) warp_sums[32] = wi;   // block total
  }
  __syncthreads();
  int res = warp_sums[warp] + incl - v;
  *total = warp_sums[32];
  return res;
}

// Context management, error plumbing and scratch buffers of libraspagpu.
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace rg
{
rg_status fail(rg_ctx* ctx, rg_status code, const std::string& msg)
{
  if (ctx) ctx->last_error = msg;
  return code;
}

rg_status checkFinite(rg_ctx* ctx, const rg_atom* atoms, long long n, const char* what)
{
  for (long long i = 0; i < n; ++i)
  {
    const rg_atom& a = atoms[i];
    if (!(std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z) && std::isfinite(a.charge) &&
          std::isfinite(a.scaling_vdw) && std::isfinite(a.scaling_coulomb)))
      return fail(ctx, RG_ERR_NONFINITE,
                  std::string(what) + ": atom " + std::to_string(i) + " has a NaN or infinite position, charge or scaling");
  }
  return RG_OK;
}

rg_status checkFiniteBox(rg_ctx* ctx, const rg_box* box, const char* what)
{
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(box->cell[i])) return fail(ctx, RG_ERR_NONFINITE, std::string(what) + ": NaN or infinite cell");
  return RG_OK;
}

bool supercellClip(const HostBox& b, double rc, double cutoff, double h[3], double ic[3][3])
{
  double w[3];
  perpendicularWidths(b, w);
  bool clip = false;
  for (int d = 0; d < 3; ++d)
  {
    const double n = std::ceil(2.0 * cutoff / w[d]);
    if (n * w[d] < 2.0 * rc) clip = true;
    h[d] = 0.5 * n * b.c[d][d];
    for (int e = 0; e < 3; ++e) ic[d][e] = b.ic[e][d] / n;
  }
  return clip;
}

rg_status cudaFail(rg_ctx* ctx, cudaError_t err, const char* what)
{
  std::string msg = std::string("CUDA error in ") + what + ": " + cudaGetErrorName(err) + " (" +
                    cudaGetErrorString(err) + ")";
  return fail(ctx, err == cudaErrorMemoryAllocation ? RG_ERR_OUT_OF_MEMORY : RG_ERR_CUDA, msg);
}

rg_status copyStream(rg_ctx* ctx, cudaStream_t* out)
{
  if (!ctx->copy_stream) RG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  *out = ctx->copy_stream;
  return RG_OK;
}

rg_status event(rg_ctx* ctx, int i, cudaEvent_t* out)
{
  while (static_cast<int>(ctx->events.size()) <= i)
  {
    cudaEvent_t e = nullptr;
    RG_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->events.push_back(e);
  }
  *out = ctx->events[i];
  return RG_OK;
}

rg_status joinCopies(rg_ctx* ctx)
{
  if (!ctx->copy_stream) return RG_OK;
  cudaEvent_t e = nullptr;
  rg_status st = event(ctx, 0, &e);
  if (st) return st;
  RG_CUDA(ctx, cudaEventRecord(e, ctx->copy_stream));
  RG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, e, 0));
  return RG_OK;
}

rg_status scratch(rg_ctx* ctx, int slot, size_t bytes, void** out)
{
  if (static_cast<int>(ctx->scratch.size()) <= slot) ctx->scratch.resize(slot + 1);
  rg_ctx::Slot& s = ctx->scratch[slot];
  if (s.bytes < bytes)
  {
    if (s.ptr)
    {
      RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      RG_CUDA(ctx, cudaFree(s.ptr));
      s.ptr = nullptr;
      s.bytes = 0;
    }
    size_t grow = bytes + bytes / 4 + 256;
    RG_CUDA(ctx, cudaMalloc(&s.ptr, grow));
    s.bytes = grow;
  }
  *out = s.ptr;
  return RG_OK;
}

rg_status pinnedScratch(rg_ctx* ctx, int slot, size_t bytes, void** out)
{
  if (static_cast<int>(ctx->pinned.size()) <= slot) ctx->pinned.resize(slot + 1);
  rg_ctx::Slot& s = ctx->pinned[slot];
  if (s.bytes < bytes)
  {
    if (s.ptr)
    {
      RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      RG_CUDA(ctx, cudaFreeHost(s.ptr));
      s.ptr = nullptr;
      s.bytes = 0;
    }
    size_t grow = bytes + bytes / 4 + 256;
    RG_CUDA(ctx, cudaMallocHost(&s.ptr, grow));
    s.bytes = grow;
  }
  *out = s.ptr;
  return RG_OK;
}

HostBox makeHostBox(const rg_box* b)
{
  HostBox box{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) box.c[c][r] = b->cell[3 * c + r];
  // double3x3::inverse (src/mathkit/double3x3.cpp:102-118)
  double m11 = box.c[0][0], m12 = box.c[1][0], m13 = box.c[2][0];
  double m21 = box.c[0][1], m22 = box.c[1][1], m23 = box.c[2][1];
  double m31 = box.c[0][2], m32 = box.c[1][2], m33 = box.c[2][2];
  double det = m11 * (m22 * m33 - m23 * m32) - m12 * (m21 * m33 - m23 * m31) + m13 * (m21 * m32 - m22 * m31);
  box.ic[0][0] = (m22 * m33 - m32 * m23) / det;
  box.ic[0][1] = -(m21 * m33 - m31 * m23) / det;
  box.ic[0][2] = (m21 * m32 - m31 * m22) / det;
  box.ic[1][0] = -(m12 * m33 - m32 * m13) / det;
  box.ic[1][1] = (m11 * m33 - m31 * m13) / det;
  box.ic[1][2] = -(m11 * m32 - m31 * m12) / det;
  box.ic[2][0] = (m12 * m23 - m22 * m13) / det;
  box.ic[2][1] = -(m11 * m23 - m21 * m13) / det;
  box.ic[2][2] = (m11 * m22 - m21 * m12) / det;
  box.volume = det;
  box.triclinic = b->triclinic != 0;
  return box;
}

void perpendicularWidths(const HostBox& b, double w[3])
{
  // SimulationBox::perpendicularWidths (src/raspakit/simulationbox.cpp:137-148)
  auto cross = [](const double* u, const double* v, double* o)
  {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
  };
  double c1[3], c2[3], c3[3];
  cross(b.c[0], b.c[1], c1);
  cross(b.c[1], b.c[2], c2);
  cross(b.c[0], b.c[2], c3);
  double v = std::fabs(b.c[0][0] * c2[0] + b.c[0][1] * c2[1] + b.c[0][2] * c2[2]);
  w[0] = v / std::sqrt(c2[0] * c2[0] + c2[1] * c2[1] + c2[2] * c2[2]);
  w[1] = v / std::sqrt(c3[0] * c3[0] + c3[1] * c3[1] + c3[2] * c3[2]);
  w[2] = v / std::sqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
}
}  // namespace rg

extern "C"
{
rg_status rg_ctx_create(int device, rg_ctx** out)
{
  if (!out) return RG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return RG_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return RG_ERR_INVALID_ARGUMENT;
  rg_ctx* ctx = new rg_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) !=
                                                  cudaSuccess)
  {
    delete ctx;
    return RG_ERR_CUDA;
  }
  ctx->stream = ctx->own_stream;
  *out = ctx;
  return RG_OK;
}

rg_status rg_ctx_destroy(rg_ctx* ctx)
{
  if (!ctx) return RG_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& s : ctx->scratch)
    if (s.ptr) cudaFree(s.ptr);
  for (auto& s : ctx->pinned)
    if (s.ptr) cudaFreeHost(s.ptr);
  if (ctx->copy_stream)
  {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return RG_OK;
}

rg_status rg_ctx_set_stream(rg_ctx* ctx, void* stream)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return RG_OK;
}

void* rg_ctx_stream(rg_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

rg_status rg_ctx_synchronize(rg_ctx* ctx)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

const char* rg_ctx_last_error(rg_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

const char* rg_version(void) { return "raspa3_b200 0.1 (sm_100a)"; }
}

// Test of a framework interpolation grid against the exact sums, on sm_100a.
//
// Replaces the grid test that System::createFrameworkInterpolationGrids (src/raspakit/system_interpolation_grids.cpp:
// 240-651, tricubic scheme) runs serially after each grid build: at random points of the simulation box it compares
// the interpolated energy and Cartesian gradient of a pseudo-atom's VDW grid with the analytical Lennard-Jones sum
// (the calculateTricubicFractionalAtPosition energy and gradient), each point weighted by exp(-beta E_vdw), and, where
// the analytical VDW energy is below the overlap criterion, the probe charge times the unit-charge Ewald grid against
// the analytical real-space Ewald sum. Energies are in K as in the reference.
//
// One thread per test point (Philox-generated, or given by the caller). The framework's periodic images within rc of
// the unit cell (the set the grid build uses) are staged tile by tile in shared memory; each thread maps its point
// into the unit cell and sums the images in FP64 (with the reference's r^2 >= 0.1 clamp). The interpolated side is the
// device interpolant with its derivative. The 36 weighted sums are reduced per block in a fixed order and the blocks
// are added in block order on the host: deterministic.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"
#include "rng.cuh"

namespace rg
{
int buildGridImages(int grid_type, const rg_forcefield* ff, const HostBox& box, const rg_atom* atoms, int n,
                    int probe_type, std::vector<double4>& pos, std::vector<double4>& par);
}

namespace
{
constexpr int kThreads = 128;
constexpr int kTile = 128;  // images staged per tile
constexpr int kSums = 36;   // 17 VDW sums, 17 charge sums, two counts (the layout of rg_grid_validation.sums)
constexpr int kHessSums = 48;  // triquintic scheme: 24 VDW and 24 charge Hessian sums (rg_grid_validation_hessian.sums)
template <int SCHEME>
constexpr int sumsOf() { return SCHEME == RG_SCHEME_TRIQUINTIC ? kSums + kHessSums : kSums; }

struct ValidateParams
{
  double uc[3][3], uic[3][3];  // unit cell and its inverse, c[col][row]
  double sc[3][3];             // simulation box
  rgd::Grid vdw, ewald;        // ewald.data null: no charge term
  const double4* vpos;         // VDW images: position, (4 eps, sigma^2, shift)
  const double4* vpar;
  const double4* epos;         // charged images: position, w = C q
  int n_vdw, n_ewald;
  double rc2, alpha, overlap, to_kelvin, charge, beta;
  long long n_points;
  const double* points;        // fractions of the simulation box (3 per point), or null: Philox
  unsigned long long seed;
  double* partial;             // [blocks][kSums]
};

__device__ __forceinline__ void accumulate(double* o, double w, double ei, double ef, const double* gi, const double* gf)
{
  o[0] += w;
  o[1] += ei * w;
  o[2] += ef * w;
  o[3] += (ef - ei) * (ef - ei) * w;
  o[4] += ef * ef * w;
#pragma unroll
  for (int a = 0; a < 3; ++a)
  {
    o[5 + a] += gi[a] * w;
    o[8 + a] += gf[a] * w;
    o[11 + a] += (gf[a] - gi[a]) * (gf[a] - gi[a]) * w;
    o[14 + a] += gf[a] * gf[a] * w;
  }
}

// Hessian sums of one term: interpolated, full, squared difference, squared full, for xx, xy, xz, yy, yz, zz
__device__ __forceinline__ void accumulateHessian(double* o, double w, const double* hi, const double* hf)
{
#pragma unroll
  for (int q = 0; q < 6; ++q)
  {
    o[q] += hi[q] * w;
    o[6 + q] += hf[q] * w;
    o[12 + q] += (hf[q] - hi[q]) * (hf[q] - hi[q]) * w;
    o[18 + q] += hf[q] * hf[q] * w;
  }
}

// H_ij += F2 dr_i dr_j + F1 delta_ij (xx, xy, xz, yy, yz, zz)
__device__ __forceinline__ void addHessian(double* h, double f1, double f2, double dx, double dy, double dz)
{
  h[0] += f2 * dx * dx + f1;
  h[1] += f2 * dx * dy;
  h[2] += f2 * dx * dz;
  h[3] += f2 * dy * dy + f1;
  h[4] += f2 * dy * dz;
  h[5] += f2 * dz * dz + f1;
}

template <int SCHEME>
__global__ void __launch_bounds__(kThreads) gridValidateKernel(ValidateParams p)
{
  constexpr bool Q = SCHEME == RG_SCHEME_TRIQUINTIC;
  constexpr int NS = sumsOf<SCHEME>();
  __shared__ double4 tpos[kTile], tpar[kTile];
  __shared__ double red[kThreads / 32][NS];
  const long long i = static_cast<long long>(blockIdx.x) * kThreads + threadIdx.x;
  const bool active = i < p.n_points;
  double u[3] = {0.5, 0.5, 0.5};
  if (active)
  {
    if (p.points)
    {
      u[0] = p.points[3 * i];
      u[1] = p.points[3 * i + 1];
      u[2] = p.points[3 * i + 2];
    }
    else
    {
      const double2 a = rgd::uniform2(p.seed, 11, i, 0), b = rgd::uniform2(p.seed, 11, i, 1);
      u[0] = a.x;
      u[1] = a.y;
      u[2] = b.x;
    }
  }
  // the point in the simulation box, and the same point mapped into the unit cell for the image sums
  double r[3], ru[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) r[a] = p.sc[0][a] * u[0] + p.sc[1][a] * u[1] + p.sc[2][a] * u[2];
  {
    double s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) s[a] = rgd::fract1(p.uic[0][a] * r[0] + p.uic[1][a] * r[1] + p.uic[2][a] * r[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) ru[a] = p.uc[0][a] * s[0] + p.uc[1][a] * s[1] + p.uc[2][a] * s[2];
  }
  // analytical Lennard-Jones energy and gradient (potentialLennardJonesTricubicDerivative: U = B - A - shift,
  // F1 = (6A - 12B)/r^2 with A = 4 eps t^3, B = A t^3; gradient = F1 * (r - r_image))
  double ev = 0.0, gv[3] = {0.0, 0.0, 0.0}, hv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int base = 0; base < p.n_vdw; base += kTile)
  {
    const int n = min(kTile, p.n_vdw - base);
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += kThreads)
    {
      tpos[j] = p.vpos[base + j];
      tpar[j] = p.vpar[base + j];
    }
    __syncthreads();
    if (active)
      for (int j = 0; j < n; ++j)
      {
        const double dx = ru[0] - tpos[j].x, dy = ru[1] - tpos[j].y, dz = ru[2] - tpos[j].z;
        const double rr = fmax(0.1, dx * dx + dy * dy + dz * dz);
        if (rr < p.rc2)
        {
          const double4 q = tpar[j];
          const double inv = 1.0 / rr;
          const double t = q.y * inv;
          const double A = q.x * t * t * t;
          const double B = A * t * t * t;
          const double f1 = (6.0 * A - 12.0 * B) * inv;
          ev += B - A - q.z;
          gv[0] += f1 * dx;
          gv[1] += f1 * dy;
          gv[2] += f1 * dz;
          // F2 = (168 B - 48 A) / r^4 (potentialLennardJonesTriquinticDerivative)
          if constexpr (Q) addHessian(hv, f1, (168.0 * B - 48.0 * A) * inv * inv, dx, dy, dz);
        }
      }
  }
  double sums[NS];
#pragma unroll
  for (int c = 0; c < NS; ++c) sums[c] = 0.0;
  double evK = 0.0, w = 0.0;
  if (active)
  {
    double gi[3], gf[3], hi[6], hf[6];
    double ei;
    if constexpr (Q)
      ei = rgd::interpolateQuinticHessian(p.vdw, r[0], r[1], r[2], gi, hi) * p.to_kelvin;
    else
      ei = rgd::interpolateGradient(p.vdw, r[0], r[1], r[2], gi) * p.to_kelvin;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      gi[a] *= p.to_kelvin;
      gf[a] = gv[a] * p.to_kelvin;
    }
    evK = ev * p.to_kelvin;
    w = exp(-p.beta * evK);
    accumulate(sums, w, ei, evK, gi, gf);
    sums[34] = 1.0;
    if constexpr (Q)
    {
#pragma unroll
      for (int q = 0; q < 6; ++q)
      {
        hi[q] *= p.to_kelvin;
        hf[q] = hv[q] * p.to_kelvin;
      }
      accumulateHessian(sums + kSums, w, hi, hf);
    }
  }
  // charge term: the unit-charge Ewald sum (potentialRealEwaldTricubicDerivative with qA = 1) times the probe charge
  if (p.ewald.data && p.charge != 0.0)
  {
    const bool take = active && evK < p.overlap;
    double ee = 0.0, ge[3] = {0.0, 0.0, 0.0}, he[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int base = 0; base < p.n_ewald; base += kTile)
    {
      const int n = min(kTile, p.n_ewald - base);
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += kThreads) tpos[j] = p.epos[base + j];
      __syncthreads();
      if (take)
        for (int j = 0; j < n; ++j)
        {
          const double dx = ru[0] - tpos[j].x, dy = ru[1] - tpos[j].y, dz = ru[2] - tpos[j].z;
          const double rr = fmax(0.1, dx * dx + dy * dy + dz * dz);
          if (rr < p.rc2)
          {
            const double rd = sqrt(rr);
            const double ec = erfc(p.alpha * rd);
            const double etr = 2.0 * p.alpha * rd * exp(-p.alpha * p.alpha * rr) * rg::kInvSqrtPi;
            const double cq = tpos[j].w;
            ee += cq * ec / rd;
            const double f1 = -cq * (etr + ec) / (rr * rd);
            ge[0] += f1 * dx;
            ge[1] += f1 * dy;
            ge[2] += f1 * dz;
            // F2 = C q (e (2 a^2 r^2 + 3) + 3 erfc) / r^5 (potentialRealEwaldTriquinticDerivative)
            if constexpr (Q)
              addHessian(he, f1,
                         cq * (etr * (2.0 * p.alpha * p.alpha * rr + 3.0) + 3.0 * ec) / (rr * rr * rd), dx, dy, dz);
          }
        }
    }
    if (take)
    {
      const double sc = p.charge * p.to_kelvin;
      double ci[3], cf[3], chi[6], chf[6];
      double eci;
      if constexpr (Q)
        eci = rgd::interpolateQuinticHessian(p.ewald, r[0], r[1], r[2], ci, chi) * sc;
      else
        eci = rgd::interpolateGradient(p.ewald, r[0], r[1], r[2], ci) * sc;
#pragma unroll
      for (int a = 0; a < 3; ++a)
      {
        ci[a] *= sc;
        cf[a] = ge[a] * sc;
      }
      accumulate(sums + 17, w, eci, ee * sc, ci, cf);
      sums[35] = 1.0;
      if constexpr (Q)
      {
#pragma unroll
        for (int q = 0; q < 6; ++q)
        {
          chi[q] *= sc;
          chf[q] = he[q] * sc;
        }
        accumulateHessian(sums + kSums + 24, w, chi, chf);
      }
    }
  }
  // fixed-order block reduction: warps by shuffles, then one thread per sum over the warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NS; ++c)
  {
    double x = sums[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp][c] = x;
  }
  __syncthreads();
  if (threadIdx.x < NS)
  {
    double x = 0.0;
    for (int wi = 0; wi < kThreads / 32; ++wi) x += red[wi][threadIdx.x];
    p.partial[static_cast<long long>(blockIdx.x) * NS + threadIdx.x] = x;
  }
}

void fillGrid(rgd::Grid& g, const double* data, int nx, int ny, int nz, const rg::HostBox& unit)
{
  g.data = data;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) g.ic[c][r] = unit.ic[c][r];
}

// Boltzmann averages and relative errors of one block of 17 sums (system_interpolation_grids.cpp:652-700)
void derive(const double* s, double* e_table, double* e_full, double* e_rel, double* g_table, double* g_full,
            double* g_rel)
{
  const double nan = std::nan("");
  *e_table = s[0] > 0.0 ? s[1] / s[0] : nan;
  *e_full = s[0] > 0.0 ? s[2] / s[0] : nan;
  *e_rel = s[4] > 0.0 ? std::sqrt(s[3] / s[4]) : nan;
  for (int a = 0; a < 3; ++a)
  {
    g_table[a] = s[0] > 0.0 ? s[5 + a] / s[0] : nan;
    g_full[a] = s[0] > 0.0 ? s[8 + a] / s[0] : nan;
    g_rel[a] = s[14 + a] > 0.0 ? std::sqrt(s[11 + a] / s[14 + a]) : nan;
  }
}
// Checks, image staging, the launch and the block-ordered sum of the partials: sumsOf<SCHEME>() values in s
template <int SCHEME>
rg_status runValidate(rg_ctx* ctx, const char* name, const rg_forcefield* ff, const rg_box* unit_cell,
                      const rg_atom* unit_atoms, int n_unit_atoms, const rg_box* simulation_box, int probe_type, int nx,
                      int ny, int nz, const double* vdw_grid_device, const double* ewald_grid_device,
                      double probe_charge, double weight_beta, int64_t n_points, uint64_t seed, const double* points,
                      std::vector<double>& s)
{
  constexpr int NS = sumsOf<SCHEME>();
  s.assign(NS, 0.0);
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  if (!ff || !unit_cell || !simulation_box || !vdw_grid_device || n_unit_atoms < 0 ||
      (n_unit_atoms > 0 && !unit_atoms) || n_points < 0)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, std::string(name) + ": null or negative argument");
  if (nx < 2 || ny < 2 || nz < 2) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, std::string(name) + ": grid shape");
  if (probe_type < 0 || probe_type >= ff->n_types)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, std::string(name) + ": probe_type out of range");
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n_points == 0) return RG_OK;

  const rg::HostBox ub = rg::makeHostBox(unit_cell), sb = rg::makeHostBox(simulation_box);
  std::vector<double4> vpos, vpar, epos, epar;
  const int nv = rg::buildGridImages(RG_GRID_LENNARD_JONES, ff, ub, unit_atoms, n_unit_atoms, probe_type, vpos, vpar);
  const bool charge = ewald_grid_device != nullptr && probe_charge != 0.0;
  const int ne = charge ? rg::buildGridImages(RG_GRID_EWALD_REAL, ff, ub, unit_atoms, n_unit_atoms, 0, epos, epar) : 0;
  const long long blocks = (n_points + kThreads - 1) / kThreads;

  // device scratch: images (slot 2), points (slot 3), block partials (slot 4); uploads staged through pinned slot 1
  const size_t img_bytes = sizeof(double4) * static_cast<size_t>(2 * nv + ne + 1);
  const size_t pts_bytes = points ? sizeof(double) * 3 * static_cast<size_t>(n_points) : 0;
  void *dimg = nullptr, *dpts = nullptr, *dpart = nullptr, *stage = nullptr;
  rg_status st = rg::scratch(ctx, 2, img_bytes, &dimg);
  if (!st && points) st = rg::scratch(ctx, 3, pts_bytes, &dpts);
  if (!st) st = rg::scratch(ctx, 4, sizeof(double) * NS * static_cast<size_t>(blocks), &dpart);
  if (st) return st;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the pinned staging slot is free
  st = rg::pinnedScratch(ctx, 1, img_bytes + pts_bytes, &stage);
  if (st) return st;
  double4* h = static_cast<double4*>(stage);
  std::memcpy(h, vpos.data(), sizeof(double4) * nv);
  std::memcpy(h + nv, vpar.data(), sizeof(double4) * nv);
  if (ne) std::memcpy(h + 2 * nv, epos.data(), sizeof(double4) * ne);
  if (points) std::memcpy(reinterpret_cast<char*>(stage) + img_bytes, points, pts_bytes);
  RG_CUDA(ctx, cudaMemcpyAsync(dimg, stage, img_bytes, cudaMemcpyHostToDevice, ctx->stream));
  if (points)
    RG_CUDA(ctx, cudaMemcpyAsync(dpts, reinterpret_cast<char*>(stage) + img_bytes, pts_bytes, cudaMemcpyHostToDevice,
                                 ctx->stream));

  ValidateParams p{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r)
    {
      p.uc[c][r] = ub.c[c][r];
      p.uic[c][r] = ub.ic[c][r];
      p.sc[c][r] = sb.c[c][r];
    }
  fillGrid(p.vdw, vdw_grid_device, nx, ny, nz, ub);
  fillGrid(p.ewald, charge ? ewald_grid_device : nullptr, nx, ny, nz, ub);
  const double4* d4 = static_cast<const double4*>(dimg);
  p.vpos = d4;
  p.vpar = d4 + nv;
  p.epos = d4 + 2 * nv;
  p.n_vdw = nv;
  p.n_ewald = ne;
  p.rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  p.alpha = ff->ewald_alpha;
  p.overlap = ff->overlap_criteria;
  p.to_kelvin = rg::energyConversionFactor() * 6.0221419947e23 / 8.314464919;  // Units::EnergyToKelvin (units.cpp)
  p.charge = charge ? probe_charge : 0.0;
  p.beta = weight_beta;
  p.n_points = n_points;
  p.points = static_cast<const double*>(dpts);
  p.seed = seed;
  p.partial = static_cast<double*>(dpart);
  gridValidateKernel<SCHEME><<<static_cast<unsigned>(blocks), kThreads, 0, ctx->stream>>>(p);
  RG_CUDA(ctx, cudaGetLastError());

  std::vector<double> part(static_cast<size_t>(blocks) * NS);
  RG_CUDA(ctx, cudaMemcpyAsync(part.data(), dpart, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (long long b = 0; b < blocks; ++b)
    for (int c = 0; c < NS; ++c) s[c] += part[static_cast<size_t>(b) * NS + c];
  return RG_OK;
}

void fillValidation(const std::vector<double>& s, rg_grid_validation* out)
{
  for (int c = 0; c < 34; ++c) out->sums[c] = s[c];
  out->n_points = static_cast<int64_t>(s[34]);
  out->n_points_charge = static_cast<int64_t>(s[35]);
  derive(s.data(), &out->energy_table, &out->energy_full, &out->energy_relative_error, out->gradient_table,
         out->gradient_full, out->gradient_relative_error);
  derive(s.data() + 17, &out->charge_energy_table, &out->charge_energy_full, &out->charge_energy_relative_error,
         out->charge_gradient_table, out->charge_gradient_full, out->charge_gradient_relative_error);
}

// Boltzmann averages and relative errors of one term's 24 Hessian sums (system_interpolation_grids.cpp:700-760)
void deriveHessian(const double* hs, double weight, double* table, double* full, double* rel)
{
  const double nan = std::nan("");
  for (int q = 0; q < 6; ++q)
  {
    table[q] = weight > 0.0 ? hs[q] / weight : nan;
    full[q] = weight > 0.0 ? hs[6 + q] / weight : nan;
    rel[q] = hs[18 + q] > 0.0 ? std::sqrt(hs[12 + q] / hs[18 + q]) : nan;
  }
}
}  // namespace

extern "C" rg_status rg_grid_validate(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell,
                                      const rg_atom* unit_atoms, int n_unit_atoms, const rg_box* simulation_box,
                                      int probe_type, int nx, int ny, int nz, const double* vdw_grid_device,
                                      const double* ewald_grid_device, double probe_charge, double weight_beta,
                                      int64_t n_points, uint64_t seed, const double* points, rg_grid_validation* out)
{
  if (ctx && !out) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_validate: null or negative argument");
  std::vector<double> s;
  rg_status st = runValidate<RG_SCHEME_TRICUBIC>(ctx, "rg_grid_validate", ff, unit_cell, unit_atoms, n_unit_atoms,
                                                 simulation_box, probe_type, nx, ny, nz, vdw_grid_device,
                                                 ewald_grid_device, probe_charge, weight_beta, n_points, seed, points,
                                                 s);
  if (st) return st;
  std::memset(out, 0, sizeof(*out));
  if (n_points > 0) fillValidation(s, out);
  return RG_OK;
}

extern "C" rg_status rg_grid_validate_triquintic(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell,
                                                 const rg_atom* unit_atoms, int n_unit_atoms,
                                                 const rg_box* simulation_box, int probe_type, int nx, int ny, int nz,
                                                 const double* vdw_grid_device, const double* ewald_grid_device,
                                                 double probe_charge, double weight_beta, int64_t n_points,
                                                 uint64_t seed, const double* points, rg_grid_validation* out,
                                                 rg_grid_validation_hessian* hessian)
{
  if (ctx && (!out || !hessian))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_validate_triquintic: null or negative argument");
  std::vector<double> s;
  rg_status st = runValidate<RG_SCHEME_TRIQUINTIC>(ctx, "rg_grid_validate_triquintic", ff, unit_cell, unit_atoms,
                                                   n_unit_atoms, simulation_box, probe_type, nx, ny, nz,
                                                   vdw_grid_device, ewald_grid_device, probe_charge, weight_beta,
                                                   n_points, seed, points, s);
  if (st) return st;
  std::memset(out, 0, sizeof(*out));
  std::memset(hessian, 0, sizeof(*hessian));
  if (n_points == 0) return RG_OK;
  fillValidation(s, out);
  for (int c = 0; c < kHessSums; ++c) hessian->sums[c] = s[kSums + c];
  deriveHessian(s.data() + kSums, s[0], hessian->hessian_table, hessian->hessian_full,
                hessian->hessian_relative_error);
  deriveHessian(s.data() + kSums + 24, s[17], hessian->charge_hessian_table, hessian->charge_hessian_full,
                hessian->charge_hessian_relative_error);
  return RG_OK;
}

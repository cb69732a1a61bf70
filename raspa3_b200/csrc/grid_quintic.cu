// Triquintic interpolation grids (27 values per grid point) on sm_100a, and device interpolation of either scheme.
//
// Replaces the triquintic branch of InterpolationEnergyGrid::makeFrameworkInterpolationGrid
// (src/raspakit/interpolation_energy_grid.cpp:3882-3962) with its per-point sums
// Interactions::calculateTriquinticFractionalAtPosition (src/raspakit/interactions/framework_molecule_grid.cpp:549-813)
// and the factor functions potentialLennardJonesTriquinticDerivative
// (src/raspakit/potentials/interpolation/triquintic_derivative_lj.ixx:33-51) and potentialRealEwaldTriquinticDerivative
// (triquintic_derivative_real_ewald.ixx:32-78).
//
// Algorithm. The same periodic-image set and brick staging as the tricubic build: a CTA owns a brick of 8 x 4 x 4 grid
// points, compacts the images within rc + R of the brick centre into shared memory, and every thread sums its point's
// 27 channels in FP64. A derivative of a radial function U(r) along directions u_1..u_n is a sum over the partial
// pairings of the directions: each pair contributes u_i.u_j, each unpaired direction u.dr, and the radial factor is
// F_{n - pairs} with F_k = (1/r d/dr)^k U. With x_a = u_a.dr for the three cell vectors, channel l of orders
// (o_x, o_y, o_z) is therefore sum_U C[l][U] F_{(n + |U|)/2} x^U over the monomials U <= o, where C holds binomials
// times pairing sums of the u_a.u_b. C depends only on the cell; it is built once on the host and travels in the launch
// parameters. A rectangular cell has u_a.u_b = 0 for a != b, which leaves 64 terms over all channels (the reference's
// per-channel formulas); a triclinic cell uses the full table, which equals the reference's full Cartesian tensors
// contracted with the cell vectors. The reference's rectangular branch deviates from the exact derivatives twice: the
// y and z first derivatives are scaled by cell[0][0] (:648-650), and the (2,2,2) channel lacks its F3 term (:671-676).
// RG_TRIQUINTIC_REFERENCE_RECTANGULAR reproduces both through the table; by default the exact values are written.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "energy.cuh"

namespace rg
{
int buildGridImages(int grid_type, const rg_forcefield* ff, const HostBox& box, const rg_atom* atoms, int n,
                    int probe_type, std::vector<double4>& pos, std::vector<double4>& par);
}

namespace
{
using rgd::quinticOrder;
constexpr int kBX = 8, kBY = 4, kBZ = 4;  // grid points per brick (one per thread)
constexpr int kThreads = kBX * kBY * kBZ;
constexpr int kPer = 2;                   // images tested per thread per staging chunk
constexpr int kChunk = kThreads * kPer;
constexpr int kSlabs = 8;                 // z-slabs of a build whose host copy overlaps the computation

template <typename Real>
struct QuinticTable
{
  Real c[27][27];  // c[channel][u_x + 3 u_y + 9 u_z]
};

struct QuinticParams
{
  double cell[3][3];  // cell[a][r]: component r of cell vector a
  double delta[3];
  double nc[3];
  int nx, ny, nz;
  int n_images;
  double rc2, filter2, alpha, overlap;
  double clip_h[3], clip_ic[3][3];  // CLIP: the supercell that the cutoff argument sizes (see grid_build.cu)
  unsigned long long* pair_count;
  double* out;
  int zb0;  // first brick along z of this launch
};

// F_k = (1/r d/dr)^k of 4 eps ((sigma^2/r^2)^6 - (sigma^2/r^2)^3) - shift, k = 0..6: the reference's factors written
// as A (c12_k t^2 - c6_k t) / r^(2k) with t = (sigma^2 / r^2)^3
template <typename Real>
__device__ __forceinline__ void ljFactors(Real rr, Real a1, Real s2, Real shift, Real F[7])
{
  const Real inv = Real(1) / rr;
  const Real q = s2 * inv;
  const Real t = q * q * q;
  const Real t2 = t * t;
  constexpr Real c12[7] = {1, -12, 168, -2688, 48384, -967680, 21288960};
  constexpr Real c6[7] = {1, -6, 48, -480, 5760, -80640, 1290240};
  F[0] = a1 * (t2 - t) - shift;
  Real ip = 1;
#pragma unroll
  for (int k = 1; k < 7; ++k)
  {
    ip *= inv;
    F[k] = a1 * (c12[k] * t2 - c6[k] * t) * ip;
  }
}

// the reference's closed forms: F_k = (-1)^k Cq (e P_k(a) + (2k-1)!! erfc(alpha r)) / r^(2k+1), a = alpha^2 r^2,
// e = 2 alpha r exp(-alpha^2 r^2) / sqrt(pi)
template <typename Real>
__device__ __forceinline__ void ewaldFactors(Real rr, Real cq, Real alpha, Real F[7])
{
  const Real r = sqrt(rr);
  const Real ec = erfc(alpha * r);
  const Real et = Real(2) * alpha * r * exp(-alpha * alpha * rr) * Real(0.564189583547756286948079451560772586);
  const Real a = alpha * alpha * rr;
  const Real inv = Real(1) / rr;
  const Real ir = Real(1) / r;
  const Real P[7] = {0,
                     1,
                     Real(2) * a + Real(3),
                     (Real(4) * a + Real(10)) * a + Real(15),
                     ((Real(8) * a + Real(28)) * a + Real(70)) * a + Real(105),
                     (((Real(16) * a + Real(72)) * a + Real(252)) * a + Real(630)) * a + Real(945),
                     ((((Real(32) * a + Real(176)) * a + Real(792)) * a + Real(2772)) * a + Real(6930)) * a +
                         Real(10395)};
  constexpr Real dfact[7] = {1, 1, 3, 15, 105, 945, 10395};
  F[0] = cq * ec * ir;
  Real ip = ir;
#pragma unroll
  for (int k = 1; k < 7; ++k)
  {
    ip *= inv;
    const Real v = cq * (et * P[k] + dfact[k] * ec) * ip;
    F[k] = (k & 1) ? -v : v;
  }
}

// Real = double: FP64 throughout. Real = float (FP32C): offsets from the brick centre rounded to FP32 once, FP32 pair
// terms, FP32 partial sums per staged chunk folded into TwoSum-compensated hi/lo pairs, FP64 epilogue.
template <typename Real, int TYPE, bool TRI, bool COUNT, bool CLIP>
__global__ void __launch_bounds__(kThreads) quinticKernel(QuinticParams p, QuinticTable<Real> tab,
                                                          const double4* __restrict__ ipos,
                                                          const double4* __restrict__ ipar)
{
  using V4 = std::conditional_t<std::is_same_v<Real, float>, float4, double4>;
  constexpr bool F32 = std::is_same_v<Real, float>;
  constexpr bool EWALD = TYPE == RG_GRID_EWALD_REAL;
  __shared__ V4 cpos[kChunk];
  __shared__ V4 cpar[EWALD ? 1 : kChunk];
  __shared__ int warp_sums[33];
  const int tid = threadIdx.x;
  const int lx = tid % kBX, ly = (tid / kBX) % kBY, lz = tid / (kBX * kBY);
  const int kb = static_cast<int>(blockIdx.z) + p.zb0;
  const int i = blockIdx.x * kBX + lx, j = blockIdx.y * kBY + ly, k = kb * kBZ + lz;
  const bool valid = i < p.nx && j < p.ny && k < p.nz;

  // grid point (interpolation_energy_grid.cpp:3827-3829) and brick centre, both from fractions of the unit cell
  const double s[3] = {i * p.delta[0], j * p.delta[1], k * p.delta[2]};
  const double sc[3] = {(blockIdx.x * kBX + 0.5 * (kBX - 1)) * p.delta[0], (blockIdx.y * kBY + 0.5 * (kBY - 1)) * p.delta[1],
                        (kb * kBZ + 0.5 * (kBZ - 1)) * p.delta[2]};
  double ctr[3];
  Real pr[3], cellR[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
  {
    const double pos = p.cell[0][r] * s[0] + p.cell[1][r] * s[1] + p.cell[2][r] * s[2];
    ctr[r] = p.cell[0][r] * sc[0] + p.cell[1][r] * sc[1] + p.cell[2][r] * sc[2];
    pr[r] = static_cast<Real>(pos - ctr[r]);
#pragma unroll
    for (int c = 0; c < 3; ++c) cellR[c][r] = static_cast<Real>(p.cell[c][r]);
  }
  const Real rc2 = static_cast<Real>(p.rc2);
  const Real alpha = static_cast<Real>(p.alpha);
  Real ch[3], cic[9];
  if constexpr (CLIP)
  {
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      ch[d] = static_cast<Real>(p.clip_h[d]);
#pragma unroll
      for (int e = 0; e < 3; ++e) cic[3 * d + e] = static_cast<Real>(p.clip_ic[d][e]);
    }
  }

  Real acc[27];                             // FP64: the sums; FP32C: the partial sums of the current chunk
  float hi[F32 ? 27 : 1], lo[F32 ? 27 : 1];  // FP32C: compensated running sums
#pragma unroll
  for (int l = 0; l < 27; ++l) acc[l] = 0;
#pragma unroll
  for (int l = 0; l < (F32 ? 27 : 1); ++l) hi[l] = lo[l] = 0.0f;
  unsigned long long npairs = 0;

  for (int base = 0; base < p.n_images; base += kChunk)
  {
    double4 ip[kPer];
    bool ok[kPer];
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q)
    {
      const int idx = base + tid * kPer + q;
      ok[q] = false;
      if (idx < p.n_images)
      {
        ip[q] = ipos[idx];
        const double dx = ip[q].x - ctr[0], dy = ip[q].y - ctr[1], dz = ip[q].z - ctr[2];
        ok[q] = dx * dx + dy * dy + dz * dz < p.filter2;
        cnt += ok[q] ? 1 : 0;
      }
    }
    int total;
    int off = blockExclusiveScan(cnt, warp_sums, &total);
#pragma unroll
    for (int q = 0; q < kPer; ++q)
      if (ok[q])
      {
        // image relative to the brick centre, in image order (deterministic sums)
        V4 c;
        c.x = static_cast<Real>(ip[q].x - ctr[0]);
        c.y = static_cast<Real>(ip[q].y - ctr[1]);
        c.z = static_cast<Real>(ip[q].z - ctr[2]);
        c.w = static_cast<Real>(ip[q].w);
        cpos[off] = c;
        if (!EWALD)
        {
          const double4 pq = ipar[base + tid * kPer + q];
          V4 pr4;
          pr4.x = static_cast<Real>(pq.x);
          pr4.y = static_cast<Real>(pq.y);
          pr4.z = static_cast<Real>(pq.z);
          pr4.w = 0;
          cpar[off] = pr4;
        }
        ++off;
      }
    __syncthreads();
    for (int c = 0; c < total; ++c)
    {
      const V4 a = cpos[c];
      // dr = posA - posB (framework_molecule_grid.cpp:575-576)
      const Real d[3] = {pr[0] - a.x, pr[1] - a.y, pr[2] - a.z};
      const Real rr = fmax(Real(0.1), d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (rr >= rc2) continue;
      if constexpr (CLIP)
        if (!rgd::insideSupercell<TRI>(ch, cic, d[0], d[1], d[2])) continue;
      if (COUNT && valid) ++npairs;
      Real F[7];
      if constexpr (EWALD)
        ewaldFactors<Real>(rr, a.w, alpha, F);
      else
      {
        const V4 pq = cpar[c];
        ljFactors<Real>(rr, pq.x, pq.y, pq.z, F);
      }
      // x_a = u_a . dr and its powers
      Real xp[3][3];
#pragma unroll
      for (int ax = 0; ax < 3; ++ax)
      {
        const Real x = TRI ? cellR[ax][0] * d[0] + cellR[ax][1] * d[1] + cellR[ax][2] * d[2] : cellR[ax][ax] * d[ax];
        xp[ax][0] = 1;
        xp[ax][1] = x;
        xp[ax][2] = x * x;
      }
#pragma unroll
      for (int l = 0; l < 27; ++l)
      {
        const int o0 = quinticOrder(l, 0), o1 = quinticOrder(l, 1), o2 = quinticOrder(l, 2);
        const int n = o0 + o1 + o2;
#pragma unroll
        for (int u2 = 0; u2 < 3; ++u2)
#pragma unroll
          for (int u1 = 0; u1 < 3; ++u1)
#pragma unroll
            for (int u0 = 0; u0 < 3; ++u0)
            {
              if (u0 > o0 || u1 > o1 || u2 > o2) continue;
              const int m = u0 + u1 + u2;
              // rectangular: only per-axis pairings (each axis keeps an even remainder); triclinic: any pairing
              if (TRI ? ((n - m) & 1) != 0 : (((o0 - u0) | (o1 - u1) | (o2 - u2)) & 1) != 0) continue;
              acc[l] += tab.c[l][u0 + 3 * u1 + 9 * u2] * (F[(n + m) / 2] * (xp[0][u0] * xp[1][u1] * xp[2][u2]));
            }
      }
    }
    if constexpr (F32)
    {
      // fold the chunk's partial sums into the compensated sums (Knuth TwoSum; the error term is exact)
#pragma unroll
      for (int l = 0; l < 27; ++l)
      {
        const float t = __fadd_rn(hi[l], acc[l]);
        const float z = __fsub_rn(t, hi[l]);
        lo[l] = __fadd_rn(lo[l], __fadd_rn(__fsub_rn(hi[l], __fsub_rn(t, z)), __fsub_rn(acc[l], z)));
        hi[l] = t;
        acc[l] = 0.0f;
      }
    }
    __syncthreads();
  }

  if (COUNT)
  {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_down_sync(0xffffffffu, npairs, o);
    if ((tid & 31) == 0 && npairs) atomicAdd(p.pair_count, npairs);
  }
  if (!valid) return;
  // derivatives per grid cell (interpolation_energy_grid.cpp:3886-3935), then the overlap clamp (:3937-3955)
  double v[27];
#pragma unroll
  for (int l = 0; l < 27; ++l)
  {
    double den = 1.0;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
      for (int q = 0; q < quinticOrder(l, ax); ++q) den *= p.nc[ax];
    const double sum = F32 ? static_cast<double>(hi[F32 ? l : 0]) + static_cast<double>(lo[F32 ? l : 0])
                           : static_cast<double>(acc[l]);
    v[l] = l == 0 ? sum : sum / den;
  }
  double* dst = p.out + 27 * (static_cast<long long>(i) + static_cast<long long>(p.nx) * (j + static_cast<long long>(p.ny) * k));
  const double oc = p.overlap;
  if (v[0] > oc)
  {
    dst[0] = 2.0 * oc;
#pragma unroll
    for (int l = 1; l < 4; ++l) dst[l] = fmin(fmax(v[l], -oc), oc);
#pragma unroll
    for (int l = 4; l < 27; ++l) dst[l] = 0.0;
  }
  else
  {
#pragma unroll
    for (int l = 0; l < 27; ++l) dst[l] = v[l];
  }
}

// Sum over the perfect pairings of a multiset of r[0] x's, r[1] y's and r[2] z's (labelled) of the product of d[a][b]
double pairings(int r0, int r1, int r2, const double d[3][3])
{
  int r[3] = {r0, r1, r2};
  int first = -1;
  for (int a = 0; a < 3 && first < 0; ++a)
    if (r[a] > 0) first = a;
  if (first < 0) return 1.0;
  --r[first];
  double sum = 0.0;
  for (int b = 0; b < 3; ++b)
  {
    if (r[b] == 0) continue;
    const double ways = static_cast<double>(r[b]);
    --r[b];
    sum += ways * d[first][b] * pairings(r[0], r[1], r[2], d);
    ++r[b];
  }
  return sum;
}

template <typename Real>
QuinticTable<Real> makeTable(const rg::HostBox& box, bool reference_rectangular)
{
  double d[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      d[a][b] = box.triclinic ? box.c[a][0] * box.c[b][0] + box.c[a][1] * box.c[b][1] + box.c[a][2] * box.c[b][2]
                              : (a == b ? box.c[a][a] * box.c[a][a] : 0.0);
  auto binom = [](int n, int k) { return (k == 0 || k == n) ? 1.0 : static_cast<double>(n); };  // n <= 2
  QuinticTable<double> t{};
  for (int l = 0; l < 27; ++l)
    for (int u2 = 0; u2 < 3; ++u2)
      for (int u1 = 0; u1 < 3; ++u1)
        for (int u0 = 0; u0 < 3; ++u0)
        {
          const int o0 = quinticOrder(l, 0), o1 = quinticOrder(l, 1), o2 = quinticOrder(l, 2);
          if (u0 > o0 || u1 > o1 || u2 > o2) continue;
          t.c[l][u0 + 3 * u1 + 9 * u2] =
              binom(o0, u0) * binom(o1, u1) * binom(o2, u2) * pairings(o0 - u0, o1 - u1, o2 - u2, d);
        }
  if (reference_rectangular && !box.triclinic)
  {
    t.c[2][3] *= box.c[0][0] / box.c[1][1];  // (0,1,0) channel, monomial x_y
    t.c[3][9] *= box.c[0][0] / box.c[2][2];  // (0,0,1) channel, monomial x_z
    t.c[26][0] = 0.0;                        // (2,2,2) channel without its F3 term
  }
  QuinticTable<Real> out{};
  for (int l = 0; l < 27; ++l)
    for (int u = 0; u < 27; ++u) out.c[l][u] = static_cast<Real>(t.c[l][u]);
  return out;
}

// bricks [p.zb0, zb1) along z
template <typename Real, int TYPE, bool TRI>
cudaError_t launchQuintic(const QuinticParams& p, int zb1, const QuinticTable<Real>& t, const double4* ipos,
                          const double4* ipar, bool count, bool clip, cudaStream_t stream)
{
  dim3 grid((p.nx + kBX - 1) / kBX, (p.ny + kBY - 1) / kBY, zb1 - p.zb0);
  if (clip)
  {
    if (count)
      quinticKernel<Real, TYPE, TRI, true, true><<<grid, kThreads, 0, stream>>>(p, t, ipos, ipar);
    else
      quinticKernel<Real, TYPE, TRI, false, true><<<grid, kThreads, 0, stream>>>(p, t, ipos, ipar);
  }
  else if (count)
    quinticKernel<Real, TYPE, TRI, true, false><<<grid, kThreads, 0, stream>>>(p, t, ipos, ipar);
  else
    quinticKernel<Real, TYPE, TRI, false, false><<<grid, kThreads, 0, stream>>>(p, t, ipos, ipar);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launchQuinticTyped(int grid_type, bool triclinic, const QuinticParams& p, int zb1,
                               const QuinticTable<Real>& t, const double4* ipos, const double4* ipar, bool count,
                               bool clip, cudaStream_t stream)
{
  if (grid_type == RG_GRID_EWALD_REAL)
    return triclinic ? launchQuintic<Real, RG_GRID_EWALD_REAL, true>(p, zb1, t, ipos, ipar, count, clip, stream)
                     : launchQuintic<Real, RG_GRID_EWALD_REAL, false>(p, zb1, t, ipos, ipar, count, clip, stream);
  return triclinic ? launchQuintic<Real, RG_GRID_LENNARD_JONES, true>(p, zb1, t, ipos, ipar, count, clip, stream)
                   : launchQuintic<Real, RG_GRID_LENNARD_JONES, false>(p, zb1, t, ipos, ipar, count, clip, stream);
}

// One thread per position: value (and gradient) of a tricubic or triquintic grid
template <int SCHEME>
__global__ void __launch_bounds__(128) interpolateKernel(rgd::Grid g, const double* __restrict__ pos, int n,
                                                         double* __restrict__ energy, double* __restrict__ grad)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double x = pos[3 * t], y = pos[3 * t + 1], z = pos[3 * t + 2];
  double gr[3];
  double e;
  if constexpr (SCHEME == RG_SCHEME_TRIQUINTIC)
    e = rgd::interpolateQuintic(g, x, y, z, grad ? gr : nullptr);
  else
    e = grad ? rgd::interpolateGradient(g, x, y, z, gr) : rgd::interpolate(g, x, y, z);
  energy[t] = e;
  if (grad)
  {
    grad[3 * t] = gr[0];
    grad[3 * t + 1] = gr[1];
    grad[3 * t + 2] = gr[2];
  }
}
}  // namespace

extern "C" rg_status rg_grid_build_triquintic(rg_ctx* ctx, int grid_type, const rg_forcefield* ff,
                                              const rg_box* unit_cell, const rg_atom* unit_atoms, int n_unit_atoms,
                                              int probe_type, double cutoff, int nx, int ny, int nz, int flags,
                                              double* out_device, double* out_host, rg_grid_stats* stats)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  if (!ff || !unit_cell || (n_unit_atoms > 0 && !unit_atoms) || n_unit_atoms < 0)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: null argument");
  if (grid_type == RG_GRID_LENNARD_JONES_REPULSION || grid_type == RG_GRID_LENNARD_JONES_ATTRACTION)
    return rg::fail(ctx, RG_ERR_UNSUPPORTED,
                    "rg_grid_build_triquintic: Lennard-Jones or Ewald-real grids only (the reference's triquintic "
                    "branch evaluates the full Lennard-Jones factor for the repulsion and attraction types)");
  if (grid_type != RG_GRID_LENNARD_JONES && grid_type != RG_GRID_EWALD_REAL)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: bad grid_type");
  if ((flags & ~(RG_TRIQUINTIC_REFERENCE_RECTANGULAR | RG_TRIQUINTIC_FP32C)) != 0)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: unknown flags");
  if (nx < 2 || ny < 2 || nz < 2)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: need >= 2 points per axis");
  if (grid_type == RG_GRID_LENNARD_JONES && (probe_type < 0 || probe_type >= ff->n_types))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: probe_type out of range");
  if (!out_device && !out_host) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: no output");
  if (!(cutoff > 0.0)) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_triquintic: cutoff must be positive");
  if (rg_status fs = rg::checkFinite(ctx, unit_atoms, n_unit_atoms, "rg_grid_build_triquintic")) return fs;
  if (rg_status fs = rg::checkFiniteBox(ctx, unit_cell, "rg_grid_build_triquintic")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));

  const rg::HostBox box = rg::makeHostBox(unit_cell);
  std::vector<double4> hpos, hpar;
  const int n_images = rg::buildGridImages(grid_type, ff, box, unit_atoms, n_unit_atoms, probe_type, hpos, hpar);
  const size_t npts = static_cast<size_t>(nx) * ny * nz;
  const size_t out_bytes = npts * 27 * sizeof(double);
  double* dout = out_device;
  void* p = nullptr;
  if (!dout)
  {
    rg_status st = rg::scratch(ctx, 0, out_bytes, &p);
    if (st) return st;
    dout = static_cast<double*>(p);
  }
  const int ni = n_images > 0 ? n_images : 1;
  rg_status st = rg::scratch(ctx, 1, 2 * sizeof(double4) * ni + 64, &p);
  if (st) return st;
  double4* dpos = static_cast<double4*>(p);
  double4* dpar = dpos + ni;
  unsigned long long* dcount = reinterpret_cast<unsigned long long*>(dpar + ni);
  if (n_images > 0)
  {
    void* hp = nullptr;
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    st = rg::pinnedScratch(ctx, 0, 2 * sizeof(double4) * n_images, &hp);
    if (st) return st;
    double4* stage = static_cast<double4*>(hp);
    std::memcpy(stage, hpos.data(), sizeof(double4) * n_images);
    std::memcpy(stage + n_images, hpar.data(), sizeof(double4) * n_images);
    RG_CUDA(ctx, cudaMemcpyAsync(dpos, stage, sizeof(double4) * n_images, cudaMemcpyHostToDevice, ctx->stream));
    RG_CUDA(ctx, cudaMemcpyAsync(dpar, stage + n_images, sizeof(double4) * n_images, cudaMemcpyHostToDevice,
                                 ctx->stream));
  }
  RG_CUDA(ctx, cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), ctx->stream));

  QuinticParams qp{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) qp.cell[c][r] = box.c[c][r];
  qp.nc[0] = nx - 1;
  qp.nc[1] = ny - 1;
  qp.nc[2] = nz - 1;
  for (int a = 0; a < 3; ++a) qp.delta[a] = 1.0 / qp.nc[a];
  qp.nx = nx;
  qp.ny = ny;
  qp.nz = nz;
  qp.n_images = n_images;
  qp.rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  double R = 0.0;  // brick half-diagonal
  for (int sx = -1; sx <= 1; sx += 2)
    for (int sy = -1; sy <= 1; sy += 2)
      for (int sz = -1; sz <= 1; sz += 2)
      {
        const double f[3] = {sx * 0.5 * (kBX - 1) * qp.delta[0], sy * 0.5 * (kBY - 1) * qp.delta[1],
                             sz * 0.5 * (kBZ - 1) * qp.delta[2]};
        double dv[3];
        rg::matvec(box.c, f, dv);
        R = std::fmax(R, std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]));
      }
  const double rf = ff->cutoff_framework_vdw + R + 1e-6;
  qp.filter2 = rf * rf;
  qp.alpha = ff->ewald_alpha;
  qp.overlap = ff->overlap_criteria;
  const bool clip = rg::supercellClip(box, ff->cutoff_framework_vdw, cutoff, qp.clip_h, qp.clip_ic);
  qp.pair_count = dcount;
  qp.out = dout;
  const bool refRect = (flags & RG_TRIQUINTIC_REFERENCE_RECTANGULAR) != 0;
  const bool fp32c = (flags & RG_TRIQUINTIC_FP32C) != 0;
  const QuinticTable<double> table64 = makeTable<double>(box, refRect);
  const QuinticTable<float> table32 = makeTable<float>(box, refRect);
  const bool count = stats != nullptr;
  // with a host output the grid is built in z-slabs and each slab's rows (contiguous in the layout) are copied on the
  // context's copy stream while the next slabs are computed
  const int zb = (nz + kBZ - 1) / kBZ;
  const int n_slabs = out_host ? std::min(zb, kSlabs) : 1;
  cudaStream_t cs = nullptr;
  if (out_host)
  {
    st = rg::copyStream(ctx, &cs);
    if (st) return st;
  }
  const size_t plane = 27 * static_cast<size_t>(nx) * ny;  // doubles per z-plane
  for (int sl = 0; sl < n_slabs; ++sl)
  {
    qp.zb0 = sl * zb / n_slabs;
    const int zb1 = (sl + 1) * zb / n_slabs;
    const cudaError_t err =
        fp32c ? launchQuinticTyped<float>(grid_type, box.triclinic, qp, zb1, table32, dpos, dpar, count, clip, ctx->stream)
              : launchQuinticTyped<double>(grid_type, box.triclinic, qp, zb1, table64, dpos, dpar, count, clip, ctx->stream);
    if (err != cudaSuccess) return rg::cudaFail(ctx, err, "quinticKernel launch");
    if (!out_host) continue;
    cudaEvent_t ev = nullptr;
    st = rg::event(ctx, 1 + sl, &ev);
    if (st) return st;
    RG_CUDA(ctx, cudaEventRecord(ev, ctx->stream));
    RG_CUDA(ctx, cudaStreamWaitEvent(cs, ev, 0));
    const size_t k0 = static_cast<size_t>(qp.zb0) * kBZ, k1 = std::min<size_t>(nz, static_cast<size_t>(zb1) * kBZ);
    if (k1 > k0)
      RG_CUDA(ctx, cudaMemcpyAsync(out_host + plane * k0, dout + plane * k0, sizeof(double) * plane * (k1 - k0),
                                   cudaMemcpyDeviceToHost, cs));
  }
  if (stats)
  {
    unsigned long long c = 0;
    RG_CUDA(ctx, cudaMemcpyAsync(&c, dcount, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    stats->pair_count = static_cast<int64_t>(c);
    stats->n_images = n_images;
    stats->h2d_bytes = static_cast<int64_t>(2 * sizeof(double4)) * n_images;
    stats->d2h_bytes = out_host ? static_cast<int64_t>(out_bytes) : 0;
  }
  if (out_host)
  {
    st = rg::joinCopies(ctx);
    if (st) return st;
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return RG_OK;
}

extern "C" rg_status rg_grid_interpolate(rg_ctx* ctx, int scheme, const double* grid_device, int nx, int ny, int nz,
                                         const rg_box* unit_cell, const double* positions, int n, double* energies,
                                         double* gradients)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  if (!grid_device || !unit_cell || n < 0 || (n > 0 && (!positions || !energies)))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_interpolate: null argument");
  if (scheme != RG_SCHEME_TRICUBIC && scheme != RG_SCHEME_TRIQUINTIC)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_interpolate: scheme must be RG_SCHEME_TRICUBIC or "
                                                  "RG_SCHEME_TRIQUINTIC");
  if (nx < 2 || ny < 2 || nz < 2) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_interpolate: grid shape");
  if (n == 0) return RG_OK;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t in_bytes = sizeof(double) * 3 * static_cast<size_t>(n);
  const size_t res_bytes = sizeof(double) * (gradients ? 4 : 1) * static_cast<size_t>(n);
  void* dp = nullptr;
  void* hp = nullptr;
  rg_status st = rg::scratch(ctx, 5, in_bytes + res_bytes, &dp);
  if (st) return st;
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the pinned slot may still feed an earlier copy
  st = rg::pinnedScratch(ctx, 1, std::max(in_bytes, res_bytes), &hp);
  if (st) return st;
  std::memcpy(hp, positions, in_bytes);
  double* dpos = static_cast<double*>(dp);
  double* dres = dpos + 3 * static_cast<size_t>(n);
  RG_CUDA(ctx, cudaMemcpyAsync(dpos, hp, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
  rgd::Grid g{grid_device, nx, ny, nz, {}};
  const rg::HostBox box = rg::makeHostBox(unit_cell);
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) g.ic[c][r] = box.ic[c][r];
  double* dgrad = gradients ? dres + n : nullptr;
  const int blocks = (n + 127) / 128;
  if (scheme == RG_SCHEME_TRIQUINTIC)
    interpolateKernel<RG_SCHEME_TRIQUINTIC><<<blocks, 128, 0, ctx->stream>>>(g, dpos, n, dres, dgrad);
  else
    interpolateKernel<RG_SCHEME_TRICUBIC><<<blocks, 128, 0, ctx->stream>>>(g, dpos, n, dres, dgrad);
  RG_CUDA(ctx, cudaGetLastError());
  RG_CUDA(ctx, cudaMemcpyAsync(hp, dres, res_bytes, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(energies, hp, sizeof(double) * n);
  if (gradients) std::memcpy(gradients, static_cast<double*>(hp) + n, sizeof(double) * 3 * static_cast<size_t>(n));
  return RG_OK;
}

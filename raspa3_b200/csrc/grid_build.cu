// (a) Rigid-framework interpolation-grid build on sm_100a.
//
// Replaces InterpolationEnergyGrid::makeFrameworkInterpolationGrid (src/raspakit/interpolation_energy_grid.cpp:
// 3800-3978) and the per-point sums of Interactions::calculateTricubicFractionalAtPosition
// (src/raspakit/interactions/framework_molecule_grid.cpp:168-282).
//
// Algorithm. The reference sums, for every grid point, over all atoms of a supercell of ceil(2 rc / width) unit
// cells with the minimum image in that supercell. Because the supercell is at least 2 rc wide, exactly one image of
// every lattice-translate class lies within rc, so that sum equals the sum over ALL periodic images of the unit-cell
// atoms with r < rc. We enumerate those images once on the host (only atoms with a nonzero parameter: eps != 0 for
// Lennard-Jones grids, q != 0 for the Ewald grid), then every CTA owns a brick of BX*BY*BZ grid points (one point per
// thread) and compacts, chunk by chunk and in image order, the images within rc + R of its brick centre (R = brick
// half-diagonal) into shared memory. All threads then stream the staged candidates (shared-memory broadcast reads)
// and accumulate energy and the seven derivative channels. Edge semantics kept from the reference: rr = max(0.1, rr),
// the strict rr < rc^2 test, fractional scaling by the cell and division by the cell counts, and the overlap clamp.
//
// Precisions: FP64 throughout; or FP32C — the point and the staged images relative to the brick centre, computed in
// FP64 and rounded to FP32 once (|offset| <= rc + R, so a displacement is off by at most ~1e-6 A), FP32 pair terms,
// FP32 partial sums per staged chunk folded into a compensated (TwoSum) hi/lo FP32 pair, and an FP64 epilogue.
// The FP32C unit-charge Ewald grid stages the images within kNearRadius + R of the brick centre in a second list and
// evaluates them in FP64: their terms (up to ~5e5 K for +2.05 e at 2.5 A) cancel to totals of a few 1e3 K, and FP32
// rounding of those few terms is what limits the energy channel otherwise.
//
// Supercell. The reference sizes its supercell with the `cutoff` argument (cutOffCoulomb for the Ewald grid,
// system_interpolation_grids.cpp:211) and tests pairs against cutOffFrameworkVDW. When that supercell is narrower
// than 2 cutOffFrameworkVDW, its minimum image drops images that lie within the pair cutoff; the CLIP kernels then
// keep a pair only if its displacement lies inside the half-open supercell box, (-1/2, 1/2] in supercell fractions.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "energy.cuh"
#include "fastmath.cuh"

namespace
{
constexpr int kPer = 2;  // images tested per thread per chunk

struct GridParams
{
  double cell[3][3];  // c[col][row]
  double delta[3];
  double ncells[3];
  int nx, ny, nz;
  int n_images;
  double rc2;
  double filter2;
  double alpha;
  double coul;
  double overlap;
  unsigned long long* pair_count;
  double* out[2];  // one output grid per Lennard-Jones probe sharing the candidate set (out[0] otherwise)
  int zb0, zb1;    // bricks along z launched: [zb0, zb1) (zb1 == 0: all)
  double near2;    // FP32C Ewald grid: images within sqrt(near2) of the brick centre are evaluated in FP64
  double clip_h[3];      // CLIP, rectangular: half the supercell lengths
  double clip_ic[3][3];  // CLIP, triclinic: supercell fractions s[d] = sum_k clip_ic[d][k] dr[k]
};

// Radius around a brick within which the FP32C Ewald grid evaluates its pair terms in FP64 (Angstrom).
#ifndef RG_GRID_NEAR_RADIUS
#define RG_GRID_NEAR_RADIUS 5.0
#endif
constexpr double kNearRadius = RG_GRID_NEAR_RADIUS;

// FP32: the hardware approximations unrefined; FP64: correctly rounded
__device__ __forceinline__ float rcpT(float x) { return rgd::rcpApprox(x); }
__device__ __forceinline__ double rcpT(double x) { return __drcp_rn(x); }
__device__ __forceinline__ double sqrtT(double x) { return sqrt(x); }
__device__ __forceinline__ double erfcT(double x) { return erfc(x); }
__device__ __forceinline__ double expT(double x) { return exp(x); }

template <typename Real>
struct Factor
{
  Real e, f1, f2, f3;
};

// potentialLennardJonesTricubicDerivative and its repulsion/attraction variants
// (src/raspakit/potentials/interpolation/tricubic_derivative_lj.ixx:33-78), written with one reciprocal.
template <int TYPE, typename Real>
__device__ __forceinline__ Factor<Real> ljFactor(Real rr, Real a1, Real s2, Real shift)
{
  Real inv = rcpT(rr);
  Real q = s2 * inv;
  Real t3 = q * q * q;
  Real t6 = t3 * t3;
  Real inv2 = inv * inv;
  Real inv3 = inv2 * inv;
  Factor<Real> f;
  if constexpr (TYPE == RG_GRID_LENNARD_JONES_REPULSION)
  {
    f.e = a1 * t6;
    f.f1 = Real(-12) * a1 * t6 * inv;
    f.f2 = Real(168) * a1 * t6 * inv2;
    f.f3 = Real(-2688) * a1 * t6 * inv3;
  }
  else if constexpr (TYPE == RG_GRID_LENNARD_JONES_ATTRACTION)
  {
    f.e = a1 * t3;
    f.f1 = Real(-6) * a1 * t3 * inv;
    f.f2 = Real(48) * a1 * t3 * inv2;
    f.f3 = Real(-480) * a1 * t3 * inv3;
  }
  else
  {
    // with A = 4 eps t3 and B = 4 eps t6: U = B - A - shift, F1 = (6A - 12B)/r^2, F2 = (168B - 48A)/r^4,
    // F3 = (480A - 2688B)/r^6 (the reference's factors, tricubic_derivative_lj.ixx:38-45, regrouped)
    const Real A = a1 * t3;
    const Real B = A * t3;
    f.e = B - A - shift;
    f.f1 = (Real(6) * A - Real(12) * B) * inv;
    f.f2 = (Real(168) * B - Real(48) * A) * inv2;
    f.f3 = (Real(480) * A - Real(2688) * B) * inv3;
  }
  return f;
}

// potentialRealEwaldTricubicDerivative with q_A = 1 (src/raspakit/potentials/interpolation/
// tricubic_derivative_real_ewald.ixx:32-56); cq = CoulombicConversionFactor * q_B.
template <typename Real>
__device__ __forceinline__ Factor<Real> ewaldFactor(Real rr, Real cq, Real alpha);

// FP32: 1/r from one reciprocal square root, erfc from the shared exp(-alpha^2 r^2)
template <>
__device__ __forceinline__ Factor<float> ewaldFactor<float>(float rr, float cq, float alpha)
{
  const float invr = rgd::rsqrtApprox(rr);
  const float r = rr * invr;
  const float ex = rgd::expApprox(-alpha * alpha * rr);
  const float ec = rgd::erfcFromExp<false>(alpha * r, ex);
  const float etr = 2.0f * alpha * r * ex * 0.564189583547756286948079451560772586f;
  const float ar2 = alpha * alpha * rr;
  const float invrr = invr * invr;
  const float i3 = invr * invrr;
  const float i5 = i3 * invrr;
  const float i7 = i5 * invrr;
  Factor<float> f;
  f.e = cq * ec * invr;
  f.f1 = -cq * (etr + ec) * i3;
  f.f2 = cq * (etr * (2.0f * ar2 + 3.0f) + 3.0f * ec) * i5;
  f.f3 = -cq * (etr * (4.0f * ar2 * ar2 + 10.0f * ar2 + 15.0f) + 15.0f * ec) * i7;
  return f;
}

template <>
__device__ __forceinline__ Factor<double> ewaldFactor<double>(double rr, double cq, double alpha)
{
  using Real = double;
  Real r = sqrtT(rr);
  Real ec = erfcT(alpha * r);
  Real ex = expT(-alpha * alpha * rr);
  Real etr = Real(2) * alpha * r * ex * Real(0.564189583547756286948079451560772586);
  Real ar2 = alpha * alpha * rr;
  Real invr = rcpT(r);
  Real invrr = invr * invr;
  Real i3 = invr * invrr;
  Real i5 = i3 * invrr;
  Real i7 = i5 * invrr;
  Factor<Real> f;
  f.e = cq * ec * invr;
  f.f1 = -cq * (etr + ec) * i3;
  f.f2 = cq * (etr * (Real(2) * ar2 + Real(3)) + Real(3) * ec) * i5;
  f.f3 = -cq * (etr * (Real(4) * ar2 * ar2 + Real(10) * ar2 + Real(15)) + Real(15) * ec) * i7;
  return f;
}

// Accumulators: FP64 plain sums, or FP32 chunk partials folded into a TwoSum-compensated hi/lo pair.
template <int N>
struct AccF64
{
  double v[N];
  __device__ void init()
  {
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = 0.0;
  }
  __device__ __forceinline__ void add(int i, double x) { v[i] += x; }
  __device__ __forceinline__ void flush() {}
  __device__ __forceinline__ double get(int i) const { return v[i]; }
};

template <int N>
struct AccF32C
{
  float p[N], hi[N], lo[N];
  __device__ void init()
  {
#pragma unroll
    for (int i = 0; i < N; ++i) p[i] = hi[i] = lo[i] = 0.0f;
  }
  __device__ __forceinline__ void add(int i, float x) { p[i] += x; }
  __device__ __forceinline__ void flush()
  {
#pragma unroll
    for (int i = 0; i < N; ++i)
    {
      // Knuth TwoSum of hi + p (exact error term), error carried in lo
      float s = __fadd_rn(hi[i], p[i]);
      float bp = __fsub_rn(s, hi[i]);
      float err = __fadd_rn(__fsub_rn(hi[i], __fsub_rn(s, bp)), __fsub_rn(p[i], bp));
      hi[i] = s;
      lo[i] = __fadd_rn(lo[i], err);
      p[i] = 0.0f;
    }
  }
  // adds an FP64 value: its FP32 head by TwoSum into hi, its FP32 tail and the TwoSum error into lo
  __device__ __forceinline__ void fold(int i, double v)
  {
    const float vh = __double2float_rn(v);
    const float vl = __double2float_rn(v - static_cast<double>(vh));
    float s = __fadd_rn(hi[i], vh);
    float bp = __fsub_rn(s, hi[i]);
    float err = __fadd_rn(__fsub_rn(hi[i], __fsub_rn(s, bp)), __fsub_rn(vh, bp));
    hi[i] = s;
    lo[i] = __fadd_rn(lo[i], __fadd_rn(err, vl));
  }
  __device__ __forceinline__ double get(int i) const { return static_cast<double>(hi[i]) + static_cast<double>(lo[i]); }
};

template <typename Real>
struct Vec4;
template <>
struct Vec4<double>
{
  using T = double4;
};
template <>
struct Vec4<float>
{
  using T = float4;
};

template <typename Real, int N>
struct AccOf;
template <int N>
struct AccOf<double, N>
{
  using T = AccF64<N>;
};
template <int N>
struct AccOf<float, N>
{
  using T = AccF32C<N>;
};

// Index of the symmetric 3-tensor component (i<=j<=k) in the 10-slot layout xxx,xxy,xxz,xyy,xyz,xzz,yyy,yyz,yzz,zzz.
__device__ __forceinline__ int sym3(int i, int j, int k)
{
  // sort
  int a = min(i, min(j, k)), c = max(i, max(j, k)), b = i + j + k - a - c;
  const int table[27] = {0, 1, 2, 0, 3, 4, 0, 0, 5, 0, 0, 0, 0, 6, 7, 0, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 9};
  return table[a * 9 + b * 3 + c];
}
__device__ __forceinline__ int sym2(int i, int j)
{
  int a = min(i, j), b = max(i, j);
  const int table[9] = {0, 1, 2, 0, 3, 4, 0, 0, 5};
  return table[a * 3 + b];
}

// Adds one pair's factors to the channels: rectangular cells need E, the gradient, the three mixed second derivatives
// and the mixed third derivative; triclinic cells the full Cartesian tensors (framework_molecule_grid.cpp:76-144) in
// symmetric storage, contracted with the cell in the epilogue.
template <bool TRICLINIC, typename Acc, typename R>
__device__ __forceinline__ void addPair(Acc& acc, const Factor<R>& f, R dx, R dy, R dz)
{
  acc.add(0, f.e);
  if constexpr (!TRICLINIC)
  {
    acc.add(1, dx * f.f1);
    acc.add(2, dy * f.f1);
    acc.add(3, dz * f.f1);
    acc.add(4, f.f2 * dx * dy);
    acc.add(5, f.f2 * dx * dz);
    acc.add(6, f.f2 * dy * dz);
    acc.add(7, f.f3 * dx * dy * dz);
  }
  else
  {
    const R d[3] = {dx, dy, dz};
    acc.add(1, dx * f.f1);
    acc.add(2, dy * f.f1);
    acc.add(3, dz * f.f1);
#pragma unroll
    for (int u = 0; u < 3; ++u)
#pragma unroll
      for (int v = u; v < 3; ++v) acc.add(4 + sym2(u, v), f.f2 * d[u] * d[v] + (u == v ? f.f1 : R(0)));
#pragma unroll
    for (int u = 0; u < 3; ++u)
#pragma unroll
      for (int v = u; v < 3; ++v)
#pragma unroll
        for (int w = v; w < 3; ++w)
          acc.add(10 + sym3(u, v, w), f.f3 * d[u] * d[v] * d[w] + (v == w ? f.f2 * d[u] : R(0)) +
                                          (u == w ? f.f2 * d[v] : R(0)) + (u == v ? f.f2 * d[w] : R(0)));
  }
}

// NP Lennard-Jones probes (1 or 2) share one candidate set: the distances, the reciprocal and the staging are computed
// once per pair and each probe adds its own factors (ipar holds NP parameter sets per image).
template <typename Real, int TYPE, bool TRICLINIC, bool COUNT, int NP, bool CLIP>
__global__ void __launch_bounds__(256, (!TRICLINIC && sizeof(Real) == 4) ? 3 : 1) gridKernel(GridParams p, const double4* __restrict__ ipos,
                                                  const double4* __restrict__ ipar, int bx, int by, int bz)
{
  using V4 = typename Vec4<Real>::T;
  constexpr bool EWALD = (TYPE == RG_GRID_EWALD_REAL);
  constexpr bool NEAR64 = EWALD && sizeof(Real) == 4;  // FP32C Ewald: FP64 list of the images near the brick
  constexpr int NCH = TRICLINIC ? 20 : 8;
  extern __shared__ unsigned char smem_raw[];
  const int nt = blockDim.x;
  const int chunk = nt * kPer;
  V4* cpos = reinterpret_cast<V4*>(smem_raw);
  V4* cpar = cpos + chunk;                                     // NP * chunk parameter sets (Lennard-Jones)
  double4* npos = reinterpret_cast<double4*>(cpos + chunk);   // near list (FP32C Ewald)
  __shared__ int warp_sums[33];

  const int tid = threadIdx.x;
  const int lx = tid % bx, ly = (tid / bx) % by, lz = tid / (bx * by);
  const int kb = static_cast<int>(blockIdx.z) + p.zb0;  // brick index along z
  const int i = blockIdx.x * bx + lx, j = blockIdx.y * by + ly, k = kb * bz + lz;
  const bool valid = (i < p.nx) && (j < p.ny) && (k < p.nz) && (lz < bz);

  // grid point (interpolation_energy_grid.cpp:3827-3829): s = (i,j,k)*delta, pos = cell * s
  double s[3] = {static_cast<double>(i) * p.delta[0], static_cast<double>(j) * p.delta[1],
                 static_cast<double>(k) * p.delta[2]};
  double pos[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) pos[r] = p.cell[0][r] * s[0] + p.cell[1][r] * s[1] + p.cell[2][r] * s[2];
  // brick centre
  double sc[3] = {(blockIdx.x * bx + 0.5 * (bx - 1)) * p.delta[0], (blockIdx.y * by + 0.5 * (by - 1)) * p.delta[1],
                  (kb * bz + 0.5 * (bz - 1)) * p.delta[2]};
  double ctr[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) ctr[r] = p.cell[0][r] * sc[0] + p.cell[1][r] * sc[1] + p.cell[2][r] * sc[2];
  // the point relative to the brick centre, computed in FP64, then in the working precision
  const Real px = static_cast<Real>(pos[0] - ctr[0]);
  const Real py = static_cast<Real>(pos[1] - ctr[1]);
  const Real pz = static_cast<Real>(pos[2] - ctr[2]);
  const Real rc2 = static_cast<Real>(p.rc2);
  const Real alpha = static_cast<Real>(p.alpha);
  Real ch[3], cic[9];
  double chd[3], cicd[9];
  if constexpr (CLIP)
  {
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      chd[d] = p.clip_h[d];
      ch[d] = static_cast<Real>(chd[d]);
#pragma unroll
      for (int e = 0; e < 3; ++e)
      {
        cicd[3 * d + e] = p.clip_ic[d][e];
        cic[3 * d + e] = static_cast<Real>(cicd[3 * d + e]);
      }
    }
  }

  typename AccOf<Real, NCH>::T accs[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) accs[q].init();
  unsigned long long npairs = 0;

  for (int base = 0; base < p.n_images; base += chunk)
  {
    // stage: each thread tests kPer consecutive images; a block scan keeps image order (deterministic sums). The far
    // and near counts travel packed in one scan (each block total is at most `chunk` < 2^16).
    double4 ip[kPer];
    bool ok[kPer], nr[kPer];
    int cnt = 0;
#pragma unroll
    for (int r = 0; r < kPer; ++r)
    {
      int idx = base + tid * kPer + r;
      ok[r] = nr[r] = false;
      if (idx < p.n_images)
      {
        ip[r] = ipos[idx];
        double dx = ip[r].x - ctr[0], dy = ip[r].y - ctr[1], dz = ip[r].z - ctr[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const bool in = d2 < p.filter2;
        nr[r] = NEAR64 && in && d2 < p.near2;
        ok[r] = in && !nr[r];
        cnt += ok[r] ? 1 : (nr[r] ? (1 << 16) : 0);
      }
    }
    int total;
    int off = blockExclusiveScan(cnt, warp_sums, &total);
    int offn = off >> 16;
    off &= 0xffff;
    const int total_near = total >> 16;
    total &= 0xffff;
#pragma unroll
    for (int r = 0; r < kPer; ++r)
    {
      const double rx = ip[r].x - ctr[0], ry = ip[r].y - ctr[1], rz = ip[r].z - ctr[2];
      if (NEAR64 && nr[r]) npos[offn++] = make_double4(rx, ry, rz, ip[r].w);
      if (ok[r])
      {
        int idx = base + tid * kPer + r;
        V4 c;
        c.x = static_cast<Real>(rx);
        c.y = static_cast<Real>(ry);
        c.z = static_cast<Real>(rz);
        c.w = static_cast<Real>(ip[r].w);
        cpos[off] = c;
        if (!EWALD)
        {
#pragma unroll
          for (int q = 0; q < NP; ++q)
          {
            const double4 pq = ipar[static_cast<long long>(idx) * NP + q];
            V4 pr;
            pr.x = static_cast<Real>(pq.x);
            pr.y = static_cast<Real>(pq.y);
            pr.z = static_cast<Real>(pq.z);
            pr.w = Real(0);
            cpar[q * chunk + off] = pr;
          }
        }
        ++off;
      }
    }
    __syncthreads();
#pragma unroll 2
    for (int c = 0; c < total; ++c)
    {
      V4 a = cpos[c];
      const Real dx = px - a.x, dy = py - a.y, dz = pz - a.z;
      Real rr = dx * dx + dy * dy + dz * dz;
      rr = rr > Real(0.1) ? rr : Real(0.1);
      bool in = rr < rc2;
      if constexpr (CLIP) in = in && rgd::insideSupercell<TRICLINIC>(ch, cic, dx, dy, dz);
      if (in)
      {
        if (COUNT && valid) ++npairs;
#pragma unroll
        for (int q = 0; q < NP; ++q)
        {
          Factor<Real> f;
          if constexpr (EWALD)
            f = ewaldFactor<Real>(rr, a.w, alpha);
          else
          {
            V4 pq = cpar[q * chunk + c];
            f = ljFactor<TYPE, Real>(rr, pq.x, pq.y, pq.z);
          }
          addPair<TRICLINIC>(accs[q], f, dx, dy, dz);
        }
      }
    }
    if constexpr (NEAR64)
    {
      // the near images: the energy in FP64 from FP64 offsets as C q (1/r - alpha erf(x)/x), x = alpha r (no erfc, no
      // exponential), folded into the compensated sums after the chunk; the derivative channels in FP32 from the
      // displacement rounded once
      double near_energy = 0.0;
      // the point's FP64 offset from the brick centre, recomputed here rather than kept live through the far loop
      double ppx, ppy, ppz;
      {
        const double si[3] = {static_cast<double>(i) * p.delta[0], static_cast<double>(j) * p.delta[1],
                              static_cast<double>(k) * p.delta[2]};
        const double sb[3] = {(blockIdx.x * bx + 0.5 * (bx - 1)) * p.delta[0],
                              (blockIdx.y * by + 0.5 * (by - 1)) * p.delta[1], (kb * bz + 0.5 * (bz - 1)) * p.delta[2]};
        double q[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
          q[r] = (p.cell[0][r] * si[0] + p.cell[1][r] * si[1] + p.cell[2][r] * si[2]) -
                 (p.cell[0][r] * sb[0] + p.cell[1][r] * sb[1] + p.cell[2][r] * sb[2]);
        ppx = q[0];
        ppy = q[1];
        ppz = q[2];
      }
      for (int c = 0; c < total_near; ++c)
      {
        const double4 a = npos[c];
        const double dx = ppx - a.x, dy = ppy - a.y, dz = ppz - a.z;
        double rr = dx * dx + dy * dy + dz * dz;
        rr = rr > 0.1 ? rr : 0.1;
        bool in = rr < p.rc2;
        if constexpr (CLIP) in = in && rgd::insideSupercell<TRICLINIC>(chd, cicd, dx, dy, dz);
        if (in)
        {
          if (COUNT && valid) ++npairs;
          const double u = p.alpha * p.alpha * rr;
          if (u <= rgd::kErfOverXMax * rgd::kErfOverXMax)
            near_energy += a.w * (rsqrt(rr) - p.alpha * rgd::erfOverX(u));
          else  // coarse grids (large bricks) only: beyond the polynomial's range
          {
            const double r = sqrt(rr);
            near_energy += a.w * erfc(p.alpha * r) / r;
          }
          Factor<Real> f = ewaldFactor<Real>(static_cast<Real>(rr), static_cast<Real>(a.w), alpha);
          f.e = Real(0);
          addPair<TRICLINIC>(accs[0], f, static_cast<Real>(dx), static_cast<Real>(dy), static_cast<Real>(dz));
        }
      }
      accs[0].flush();
      accs[0].fold(0, near_energy);
    }
    else
    {
#pragma unroll
      for (int q = 0; q < NP; ++q) accs[q].flush();
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

#pragma unroll
  for (int q = 0; q < NP; ++q)
  {
  const auto& acc = accs[q];
  double v[8];
  v[0] = acc.get(0);
  if constexpr (!TRICLINIC)
  {
    // rectangular scaling by the cell diagonal (framework_molecule_grid.cpp:236-243)
    const double cx = p.cell[0][0], cy = p.cell[1][1], cz = p.cell[2][2];
    v[1] = acc.get(1) * cx;
    v[2] = acc.get(2) * cy;
    v[3] = acc.get(3) * cz;
    v[4] = acc.get(4) * cx * cy;
    v[5] = acc.get(5) * cx * cz;
    v[6] = acc.get(6) * cy * cz;
    v[7] = acc.get(7) * cx * cy * cz;
  }
  else
  {
    // contraction with the cell vectors (framework_molecule_grid.cpp:244-279)
    double g[3] = {acc.get(1), acc.get(2), acc.get(3)};
    double f0 = 0, f1 = 0, f2 = 0, s01 = 0, s02 = 0, s12 = 0, t012 = 0;
    for (int a = 0; a < 3; ++a)
    {
      f0 += p.cell[0][a] * g[a];
      f1 += p.cell[1][a] * g[a];
      f2 += p.cell[2][a] * g[a];
      for (int b = 0; b < 3; ++b)
      {
        double h = acc.get(4 + sym2(a, b));
        s01 += p.cell[0][a] * p.cell[1][b] * h;
        s02 += p.cell[0][a] * p.cell[2][b] * h;
        s12 += p.cell[1][a] * p.cell[2][b] * h;
        for (int c = 0; c < 3; ++c) t012 += p.cell[0][a] * p.cell[1][b] * p.cell[2][c] * acc.get(10 + sym3(a, b, c));
      }
    }
    v[1] = f0;
    v[2] = f1;
    v[3] = f2;
    v[4] = s01;
    v[5] = s02;
    v[6] = s12;
    v[7] = t012;
  }
  // division by the cell counts and the overlap clamp (interpolation_energy_grid.cpp:3847-3874)
  v[1] /= p.ncells[0];
  v[2] /= p.ncells[1];
  v[3] /= p.ncells[2];
  v[4] /= p.ncells[0] * p.ncells[1];
  v[5] /= p.ncells[0] * p.ncells[2];
  v[6] /= p.ncells[1] * p.ncells[2];
  v[7] /= p.ncells[0] * p.ncells[1] * p.ncells[2];
  const double oc = p.overlap;
  if (v[0] > oc)
  {
    v[0] = 2.0 * oc;
    v[1] = fmin(fmax(v[1], -oc), oc);
    v[2] = fmin(fmax(v[2], -oc), oc);
    v[3] = fmin(fmax(v[3], -oc), oc);
    v[4] = v[5] = v[6] = v[7] = 0.0;
  }
  double2* dst = reinterpret_cast<double2*>(p.out[q] + 8 * (static_cast<long long>(i) +
                                                         static_cast<long long>(p.nx) *
                                                             (static_cast<long long>(j) + static_cast<long long>(p.ny) * k)));
  dst[0] = make_double2(v[0], v[1]);
  dst[1] = make_double2(v[2], v[3]);
  dst[2] = make_double2(v[4], v[5]);
  dst[3] = make_double2(v[6], v[7]);
  }
}

// ---------------------------------------------------------------------------------------------------------------------
// FP32C rectangular grids with packed FP32 arithmetic (sm_100a f32x2 FMA / multiply / add).
//
// Each thread owns two grid points of its brick column, two planes apart along z: (i, j, k) and (i, j, k + 2) in a
// brick of 8 x 8 x 4 points (128 threads). The two points share dx and dy to every staged image, and every operation
// after dz is one packed instruction for both pairs; the reciprocal, reciprocal square root and base-2 exponential
// stay scalar. Each warp compacts the staged images within reach of its own 8 x 4 x 2 points into an index list and
// runs over it without branches (independent iterations the compiler can interleave): a lane whose pair is outside
// the cutoff is masked by zeroing its parameters, so its factors and terms are exactly 0.
// FP32 partial sums per staged chunk are added into FP64 sums kept in shared memory. The unit-charge Ewald grid keeps
// the near-image list of gridKernel: images within kNearRadius + R of the brick centre, energy in FP64.
// ---------------------------------------------------------------------------------------------------------------------
constexpr int kPackThreads = 128;
// images staged per thread and chunk: 4 for the Ewald kernel; for Lennard-Jones kernels RG_PACK_PER_LJ (their two
// parameter lists and the sums of two probes would otherwise hold them to 3 CTAs per SM)
#ifndef RG_PACK_PER_LJ
#define RG_PACK_PER_LJ 2
#endif
template <int TYPE>
constexpr int packPer()
{
  return TYPE == RG_GRID_EWALD_REAL ? 4 : RG_PACK_PER_LJ;
}
// candidate iterations unrolled in the packed kernels (measured on B200: 3 for the Ewald kernel, 4 for Lennard-Jones)
constexpr int kPackUnrollEwald = 3;
constexpr int kPackUnrollLJ = 4;

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

struct Factor2
{
  float2 e, f1, f2, f3;
};

// ewaldFactor<float> for two pairs; cq is zero on a masked lane. The first- and third-derivative factors come out with
// their signs flipped (f1 = C q (etr + ec) / r^3 and f3 = C q (etr (4 a^2 + 10 a + 15) + 15 ec) / r^7, a = alpha^2 r^2,
// both positive): the channels they feed are negated once when the chunk's sums are folded into FP64.
struct EwaldConst
{
  float2 g, half_alpha, etr, two_a2, four_a4, ten_a2;
};
__device__ __forceinline__ EwaldConst ewaldConst(float alpha)
{
  const float a2 = alpha * alpha;
  EwaldConst c;
  c.g = bc(-a2 * 1.4426950408889634f);           // exp(-alpha^2 r^2) = 2^(g r^2)
  c.half_alpha = bc(0.5f * alpha);
  c.etr = bc(alpha * 1.1283791670955126f);       // 2 alpha / sqrt(pi)
  c.two_a2 = bc(2.0f * a2);
  c.four_a4 = bc(4.0f * a2 * a2);
  c.ten_a2 = bc(10.0f * a2);
  return c;
}
__device__ __forceinline__ Factor2 ewaldFactor2(float2 rr, float2 cq, const EwaldConst& k)
{
  const float2 invr = make_float2(rgd::rsqrtApprox(rr.x), rgd::rsqrtApprox(rr.y));
  const float2 r = mul2(rr, invr);
  const float2 g = mul2(rr, k.g);
  float2 ex;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ex.x) : "f"(g.x));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ex.y) : "f"(g.y));
  const float2 tden = fma2(r, k.half_alpha, bc(1.0f));
  const float2 t = make_float2(rgd::rcpApprox(tden.x), rgd::rcpApprox(tden.y));
  // rgd::erfcFromExp's polynomial in t, packed
  float2 R = bc(-0.02496027760207653f);
  R = fma2(R, t, bc(0.09420006722211838f));
  R = fma2(R, t, bc(-0.024484887719154358f));
  R = fma2(R, t, bc(-0.36430737376213074f));
  R = fma2(R, t, bc(0.534475564956665f));
  R = fma2(R, t, bc(-0.11705945432186127f));
  R = fma2(R, t, bc(0.3620023727416992f));
  R = fma2(R, t, bc(0.25453805923461914f));
  R = fma2(R, t, bc(0.2858136296272278f));
  R = fma2(R, t, bc(-0.00021772264153696597f));
  const float2 ec = mul2(ex, R);                 // erfc(alpha r)
  const float2 etr = mul2(mul2(r, ex), k.etr);   // 2 alpha r exp(-alpha^2 r^2) / sqrt(pi)
  const float2 q1 = mul2(cq, invr);              // C q / r
  const float2 i2 = mul2(invr, invr);
  const float2 s1 = mul2(q1, i2);
  const float2 s2 = mul2(s1, i2);
  const float2 s3 = mul2(s2, i2);
  const float2 ec3 = mul2(ec, bc(3.0f));
  Factor2 f;
  f.e = mul2(ec, q1);
  f.f1 = mul2(add2(etr, ec), s1);
  f.f2 = mul2(fma2(etr, fma2(rr, k.two_a2, bc(3.0f)), ec3), s2);
  f.f3 = mul2(fma2(etr, fma2(fma2(rr, k.four_a4, k.ten_a2), rr, bc(15.0f)), mul2(ec3, bc(5.0f))), s3);
  return f;
}

// ljFactor for two pairs from the shared reciprocals; a1 and shift are zero on a masked lane
template <int TYPE>
__device__ __forceinline__ Factor2 ljFactor2(float2 inv, float2 inv2, float2 inv3, float2 a1, float s2, float2 shift)
{
  const float2 q = mul2(inv, bc(s2));
  const float2 t3 = mul2(mul2(q, q), q);
  Factor2 f;
  if constexpr (TYPE == RG_GRID_LENNARD_JONES_REPULSION)
  {
    const float2 B = mul2(mul2(a1, t3), t3);
    f.e = B;
    f.f1 = mul2(mul2(B, bc(-12.0f)), inv);
    f.f2 = mul2(mul2(B, bc(168.0f)), inv2);
    f.f3 = mul2(mul2(B, bc(-2688.0f)), inv3);
  }
  else if constexpr (TYPE == RG_GRID_LENNARD_JONES_ATTRACTION)
  {
    const float2 A = mul2(a1, t3);
    f.e = A;
    f.f1 = mul2(mul2(A, bc(-6.0f)), inv);
    f.f2 = mul2(mul2(A, bc(48.0f)), inv2);
    f.f3 = mul2(mul2(A, bc(-480.0f)), inv3);
  }
  else
  {
    const float2 A = mul2(a1, t3);
    const float2 B = mul2(A, t3);
    f.e = add2(fma2(A, bc(-1.0f), B), mul2(shift, bc(-1.0f)));
    f.f1 = mul2(fma2(A, bc(6.0f), mul2(B, bc(-12.0f))), inv);
    f.f2 = mul2(fma2(B, bc(168.0f), mul2(A, bc(-48.0f))), inv2);
    f.f3 = mul2(fma2(A, bc(480.0f), mul2(B, bc(-2688.0f))), inv3);
  }
  return f;
}

// the 8 rectangular channels of both points: E, dx f1, dy f1, dz f1, f2 dx dy, f2 dx dz, f2 dy dz, f3 dx dy dz
template <bool ENERGY>
__device__ __forceinline__ void addPair2(float2 (&P)[8], const Factor2& f, float dx, float dy, float2 dz)
{
  if constexpr (ENERGY) P[0] = add2(P[0], f.e);
  P[1] = fma2(bc(dx), f.f1, P[1]);
  P[2] = fma2(bc(dy), f.f1, P[2]);
  P[3] = fma2(dz, f.f1, P[3]);
  const float dxy = dx * dy;
  P[4] = fma2(bc(dxy), f.f2, P[4]);
  P[5] = fma2(mul2(bc(dx), dz), f.f2, P[5]);
  P[6] = fma2(mul2(bc(dy), dz), f.f2, P[6]);
  P[7] = fma2(mul2(bc(dxy), dz), f.f3, P[7]);
}

// FP64 energy of a near image: C q erfc(alpha r) / r as C q (1/r - alpha erf(x)/x), x = alpha r, or erfc directly
// beyond the polynomial's range (coarse grids only)
__device__ __forceinline__ double nearEwaldEnergy(double rr, double cq, double alpha)
{
  const double u = alpha * alpha * rr;
  if (u <= rgd::kErfOverXMax * rgd::kErfOverXMax) return cq * (rsqrt(rr) - alpha * rgd::erfOverX(u));
  const double r = sqrt(rr);
  return cq * erfc(alpha * r) / r;
}

template <int TYPE, int NP, bool COUNT>
__global__ void __launch_bounds__(kPackThreads, 4) gridKernelPacked(GridParams p, const double4* __restrict__ ipos,
                                                                   const double4* __restrict__ ipar)
{
  constexpr bool EWALD = (TYPE == RG_GRID_EWALD_REAL);
  constexpr int kPackPer = packPer<TYPE>();
  constexpr int kPackChunk = kPackThreads * kPackPer;
  constexpr int kSlots = NP * 8 * 2;  // FP64 sums: [probe][channel][point]
  extern __shared__ unsigned char smem_raw[];
  float4* cpos = reinterpret_cast<float4*>(smem_raw);
  float4* cpar = cpos + kPackChunk;                              // Lennard-Jones: NP parameter lists
  double4* npos = reinterpret_cast<double4*>(cpos + kPackChunk);  // Ewald: near list
  double* sums = reinterpret_cast<double*>(smem_raw + sizeof(float4) * kPackChunk *
                                                         (EWALD ? 3 : 1 + NP));  // [slot][thread]
  __shared__ int warp_sums[33];
  __shared__ unsigned short wlists[(kPackThreads / 32) * kPackChunk];  // per warp: indices of its candidates

  const int tid = threadIdx.x;
  const int lx = tid & 7, ly = (tid >> 3) & 7, lz = tid >> 6;
  const int kb = static_cast<int>(blockIdx.z) + p.zb0;
  const int i = blockIdx.x * 8 + lx, j = blockIdx.y * 8 + ly;
  const int k0 = kb * 4 + lz, k1 = k0 + 2;
  const bool valid0 = i < p.nx && j < p.ny && k0 < p.nz;
  const bool valid1 = i < p.nx && j < p.ny && k1 < p.nz;

  // the points and the brick centre (rectangular: the cell diagonal), relative offsets computed in FP64
  const double cx = p.cell[0][0], cy = p.cell[1][1], cz = p.cell[2][2];
  const double ctr[3] = {(blockIdx.x * 8 + 3.5) * p.delta[0] * cx, (blockIdx.y * 8 + 3.5) * p.delta[1] * cy,
                         (kb * 4 + 1.5) * p.delta[2] * cz};
  const double qx = i * p.delta[0] * cx - ctr[0], qy = j * p.delta[1] * cy - ctr[1];
  const double qz0 = k0 * p.delta[2] * cz - ctr[2], qz1 = k1 * p.delta[2] * cz - ctr[2];
  const float px = static_cast<float>(qx), py = static_cast<float>(qy);
  const float2 pz = make_float2(static_cast<float>(qz0), static_cast<float>(qz1));
  const float rc2 = static_cast<float>(p.rc2);
  const EwaldConst ek = ewaldConst(static_cast<float>(p.alpha));
  // the warp's points: x in [0, 7], y in [4 (warp & 1), + 3], z in {lz, lz + 2} (grid steps within the brick); its
  // box centre relative to the brick centre and its half-diagonal R_w, plus a margin for FP32 rounding
  const int warp = tid >> 5, lane = tid & 31;
  const double hx = p.delta[0] * cx, hy = p.delta[1] * cy, hz = p.delta[2] * cz;
  const float3 wc = make_float3(0.0f, static_cast<float>((4 * (warp & 1) - 2) * hy),
                                static_cast<float>(((warp >> 1) - 0.5) * hz));
  const double rw = sqrt(p.rc2) + sqrt(12.25 * hx * hx + 2.25 * hy * hy + hz * hz) + 1e-3;
  const float rw2 = static_cast<float>(rw * rw);
  unsigned short* wl = wlists + warp * kPackChunk;

#pragma unroll
  for (int s = 0; s < kSlots; ++s) sums[s * kPackThreads + tid] = 0.0;
  unsigned long long npairs = 0;

  for (int base = 0; base < p.n_images; base += kPackChunk)
  {
    double4 ip[kPackPer];
    bool ok[kPackPer], nr[kPackPer];
    int cnt = 0;
#pragma unroll
    for (int r = 0; r < kPackPer; ++r)
    {
      const int idx = base + tid * kPackPer + r;
      ok[r] = nr[r] = false;
      if (idx < p.n_images)
      {
        ip[r] = ipos[idx];
        const double dx = ip[r].x - ctr[0], dy = ip[r].y - ctr[1], dz = ip[r].z - ctr[2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const bool in = d2 < p.filter2;
        nr[r] = EWALD && in && d2 < p.near2;
        ok[r] = in && !nr[r];
        cnt += ok[r] ? 1 : (nr[r] ? (1 << 16) : 0);
      }
    }
    int total;
    int off = blockExclusiveScan(cnt, warp_sums, &total);
    int offn = off >> 16;
    off &= 0xffff;
    const int total_near = total >> 16;
    total &= 0xffff;
#pragma unroll
    for (int r = 0; r < kPackPer; ++r)
    {
      const double rx = ip[r].x - ctr[0], ry = ip[r].y - ctr[1], rz = ip[r].z - ctr[2];
      if (EWALD && nr[r]) npos[offn++] = make_double4(rx, ry, rz, ip[r].w);
      if (ok[r])
      {
        cpos[off] = make_float4(static_cast<float>(rx), static_cast<float>(ry), static_cast<float>(rz),
                                static_cast<float>(ip[r].w));
        if constexpr (!EWALD)
        {
          const long long idx = base + tid * kPackPer + r;
#pragma unroll
          for (int q = 0; q < NP; ++q)
          {
            const double4 pq = ipar[idx * NP + q];
            cpar[q * kPackChunk + off] =
                make_float4(static_cast<float>(pq.x), static_cast<float>(pq.y), static_cast<float>(pq.z), 0.0f);
          }
        }
        ++off;
      }
    }
    __syncthreads();

    // this warp's candidates: the staged images within rc + R_w of the warp's own point box (a superset of those within
    // rc of any of its points), indices in staging order
    int nw = 0;
    for (int b0 = 0; b0 < total; b0 += 32)
    {
      const int c = b0 + lane;
      bool in = false;
      if (c < total)
      {
        const float4 a = cpos[c];
        const float ex = a.x - wc.x, ey = a.y - wc.y, ez = a.z - wc.z;
        in = fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < rw2;
      }
      const unsigned ballot = __ballot_sync(0xffffffffu, in);
      if (in) wl[nw + __popc(ballot & ((1u << lane) - 1u))] = static_cast<unsigned short>(c);
      nw += __popc(ballot);
    }
    __syncwarp();

    // every candidate of the list for both points of every lane, branch-free: a lane whose pair is outside the cutoff
    // has its charge (Ewald) or its epsilon and shift (Lennard-Jones) zeroed, so its factors and terms are exactly 0
    float2 P[NP][8];
#pragma unroll
    for (int q = 0; q < NP; ++q)
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) P[q][ch] = bc(0.0f);
    constexpr int kUnroll = EWALD ? kPackUnrollEwald : kPackUnrollLJ;
#pragma unroll kUnroll
    for (int w = 0; w < nw; ++w)
    {
      const int c = wl[w];
      const float4 a = cpos[c];
      const float dx = px - a.x, dy = py - a.y;
      const float2 dz = add2(pz, bc(-a.z));
      float2 rr = fma2(dz, dz, bc(fmaf(dx, dx, dy * dy)));
      rr.x = fmaxf(rr.x, 0.1f);
      rr.y = fmaxf(rr.y, 0.1f);
      const bool in0 = rr.x < rc2, in1 = rr.y < rc2;
      if (COUNT) npairs += (in0 && valid0 ? 1 : 0) + (in1 && valid1 ? 1 : 0);
      if constexpr (EWALD)
      {
        const Factor2 f = ewaldFactor2(rr, make_float2(in0 ? a.w : 0.0f, in1 ? a.w : 0.0f), ek);
        addPair2<true>(P[0], f, dx, dy, dz);
      }
      else
      {
        const float2 inv = make_float2(rgd::rcpApprox(rr.x), rgd::rcpApprox(rr.y));
        const float2 inv2 = mul2(inv, inv);
        const float2 inv3 = mul2(inv2, inv);
#pragma unroll
        for (int q = 0; q < NP; ++q)
        {
          const float4 pq = cpar[q * kPackChunk + c];
          const Factor2 f = ljFactor2<TYPE>(inv, inv2, inv3, make_float2(in0 ? pq.x : 0.0f, in1 ? pq.x : 0.0f),
                                            pq.y, make_float2(in0 ? pq.z : 0.0f, in1 ? pq.z : 0.0f));
          addPair2<true>(P[q], f, dx, dy, dz);
        }
      }
    }
    double ne0 = 0.0, ne1 = 0.0;
    if constexpr (EWALD)
    {
      // near images: energy in FP64 from FP64 offsets, derivative channels packed in FP32 from the exact
      // displacement rounded once
      for (int c = 0; c < total_near; ++c)
      {
        const double4 a = npos[c];
        const double dx = qx - a.x, dy = qy - a.y, dz0 = qz0 - a.z, dz1 = qz1 - a.z;
        const double dxy = dx * dx + dy * dy;
        const double rr0 = fmax(dxy + dz0 * dz0, 0.1), rr1 = fmax(dxy + dz1 * dz1, 0.1);
        const bool in0 = rr0 < p.rc2, in1 = rr1 < p.rc2;
        if (in0 || in1)
        {
          if (COUNT) npairs += (in0 && valid0 ? 1 : 0) + (in1 && valid1 ? 1 : 0);
          if (in0) ne0 += nearEwaldEnergy(rr0, a.w, p.alpha);
          if (in1) ne1 += nearEwaldEnergy(rr1, a.w, p.alpha);
          const float cq = static_cast<float>(a.w);
          const Factor2 f = ewaldFactor2(make_float2(static_cast<float>(rr0), static_cast<float>(rr1)),
                                         make_float2(in0 ? cq : 0.0f, in1 ? cq : 0.0f), ek);
          addPair2<false>(P[0], f, static_cast<float>(dx), static_cast<float>(dy),
                          make_float2(static_cast<float>(dz0), static_cast<float>(dz1)));
        }
      }
    }
    // the chunk's FP32 partial sums into the FP64 sums
#pragma unroll
    for (int q = 0; q < NP; ++q)
#pragma unroll
      for (int ch = 0; ch < 8; ++ch)
      {
        const int s = (q * 8 + ch) * 2;
        double e0 = static_cast<double>(P[q][ch].x), e1 = static_cast<double>(P[q][ch].y);
        if (EWALD && ch == 0)
        {
          e0 += ne0;
          e1 += ne1;
        }
        if (EWALD && (ch == 1 || ch == 2 || ch == 3 || ch == 7))
        {
          e0 = -e0;  // ewaldFactor2's sign-flipped f1 and f3
          e1 = -e1;
        }
        sums[s * kPackThreads + tid] += e0;
        sums[(s + 1) * kPackThreads + tid] += e1;
      }
    __syncthreads();
  }

  if (COUNT)
  {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_down_sync(0xffffffffu, npairs, o);
    if ((tid & 31) == 0 && npairs) atomicAdd(p.pair_count, npairs);
  }
#pragma unroll
  for (int q = 0; q < NP; ++q)
#pragma unroll
    for (int pt = 0; pt < 2; ++pt)
    {
      if (!(pt == 0 ? valid0 : valid1)) continue;
      const int k = pt == 0 ? k0 : k1;
      double v[8];
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) v[ch] = sums[((q * 8 + ch) * 2 + pt) * kPackThreads + tid];
      // rectangular scaling by the cell diagonal and division by the cell counts (framework_molecule_grid.cpp:236-243,
      // interpolation_energy_grid.cpp:3847-3856), then the overlap clamp (:3858-3874)
      v[1] *= cx / p.ncells[0];
      v[2] *= cy / p.ncells[1];
      v[3] *= cz / p.ncells[2];
      v[4] *= cx * cy / (p.ncells[0] * p.ncells[1]);
      v[5] *= cx * cz / (p.ncells[0] * p.ncells[2]);
      v[6] *= cy * cz / (p.ncells[1] * p.ncells[2]);
      v[7] *= cx * cy * cz / (p.ncells[0] * p.ncells[1] * p.ncells[2]);
      const double oc = p.overlap;
      if (v[0] > oc)
      {
        v[0] = 2.0 * oc;
        v[1] = fmin(fmax(v[1], -oc), oc);
        v[2] = fmin(fmax(v[2], -oc), oc);
        v[3] = fmin(fmax(v[3], -oc), oc);
        v[4] = v[5] = v[6] = v[7] = 0.0;
      }
      double2* dst = reinterpret_cast<double2*>(
          p.out[q] + 8 * (static_cast<long long>(i) +
                          static_cast<long long>(p.nx) * (static_cast<long long>(j) + static_cast<long long>(p.ny) * k)));
      dst[0] = make_double2(v[0], v[1]);
      dst[1] = make_double2(v[2], v[3]);
      dst[2] = make_double2(v[4], v[5]);
      dst[3] = make_double2(v[6], v[7]);
    }
}

template <int TYPE, int NP>
size_t packedSharedBytes()
{
  constexpr bool EWALD = TYPE == RG_GRID_EWALD_REAL;
  return sizeof(float4) * kPackThreads * packPer<TYPE>() * (EWALD ? 3 : 1 + NP) + sizeof(double) * NP * 16 * kPackThreads;
}

template <int TYPE, int NP, bool COUNT>
cudaError_t launchPacked(const GridParams& p, const double4* ipos, const double4* ipar, cudaStream_t stream)
{
  const int zbricks = p.zb1 > p.zb0 ? p.zb1 - p.zb0 : (p.nz + 3) / 4;
  dim3 grid((p.nx + 7) / 8, (p.ny + 7) / 8, zbricks);
  const size_t shmem = packedSharedBytes<TYPE, NP>();
  auto kern = gridKernelPacked<TYPE, NP, COUNT>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shmem));
  kern<<<grid, kPackThreads, shmem, stream>>>(p, ipos, ipar);
  return cudaGetLastError();
}

// Dynamic shared memory of a launch: the FP32/FP64 candidate list, NP parameter lists for Lennard-Jones grids, and the
// FP64 near list of the FP32C Ewald grid.
template <typename Real, int TYPE, int NP>
size_t gridSharedBytes(int nt)
{
  const size_t chunk = static_cast<size_t>(nt) * kPer;
  size_t b = sizeof(typename Vec4<Real>::T) * chunk;
  if (TYPE != RG_GRID_EWALD_REAL) b += NP * sizeof(typename Vec4<Real>::T) * chunk;
  if (TYPE == RG_GRID_EWALD_REAL && sizeof(Real) == 4) b += sizeof(double4) * chunk;
  return b;
}

template <typename Real, int TYPE, bool TRI, int NP, bool COUNT, bool CLIP>
cudaError_t launchKernel(const GridParams& p, const double4* ipos, const double4* ipar, int bx, int by, int bz,
                         cudaStream_t stream)
{
  const int zbricks = p.zb1 > p.zb0 ? p.zb1 - p.zb0 : (p.nz + bz - 1) / bz;
  dim3 grid((p.nx + bx - 1) / bx, (p.ny + by - 1) / by, zbricks);
  const int nt = bx * by * bz;
  const size_t shmem = gridSharedBytes<Real, TYPE, NP>(nt);
  auto kern = gridKernel<Real, TYPE, TRI, COUNT, NP, CLIP>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shmem));
  kern<<<grid, nt, shmem, stream>>>(p, ipos, ipar, bx, by, bz);
  return cudaGetLastError();
}

template <typename Real, int TYPE, bool TRI, int NP = 1>
cudaError_t launchTyped(const GridParams& p, const double4* ipos, const double4* ipar, int bx, int by, int bz,
                        bool count, bool clip, cudaStream_t stream)
{
  // FP32C rectangular grids (cell diagonal only) without a supercell clip: the packed two-point kernel (bricks of
  // 8 x 8 x 4 points)
  if constexpr (sizeof(Real) == 4 && !TRI)
    if (!clip && bx == 8 && by == 8 && bz == 4 && p.cell[0][1] == 0.0 && p.cell[0][2] == 0.0 && p.cell[1][0] == 0.0 &&
        p.cell[1][2] == 0.0 && p.cell[2][0] == 0.0 && p.cell[2][1] == 0.0)
      return count ? launchPacked<TYPE, NP, true>(p, ipos, ipar, stream)
                   : launchPacked<TYPE, NP, false>(p, ipos, ipar, stream);
  if (clip)
    return count ? launchKernel<Real, TYPE, TRI, NP, true, true>(p, ipos, ipar, bx, by, bz, stream)
                 : launchKernel<Real, TYPE, TRI, NP, false, true>(p, ipos, ipar, bx, by, bz, stream);
  return count ? launchKernel<Real, TYPE, TRI, NP, true, false>(p, ipos, ipar, bx, by, bz, stream)
               : launchKernel<Real, TYPE, TRI, NP, false, false>(p, ipos, ipar, bx, by, bz, stream);
}

template <typename Real, bool TRI>
cudaError_t launchPrec(int type, const GridParams& p, const double4* ipos, const double4* ipar, int bx, int by, int bz,
                       bool count, bool clip, cudaStream_t stream)
{
  switch (type)
  {
    case RG_GRID_LENNARD_JONES:
      return launchTyped<Real, RG_GRID_LENNARD_JONES, TRI>(p, ipos, ipar, bx, by, bz, count, clip, stream);
    case RG_GRID_EWALD_REAL:
      return launchTyped<Real, RG_GRID_EWALD_REAL, TRI>(p, ipos, ipar, bx, by, bz, count, clip, stream);
    case RG_GRID_LENNARD_JONES_REPULSION:
      return launchTyped<Real, RG_GRID_LENNARD_JONES_REPULSION, TRI>(p, ipos, ipar, bx, by, bz, count, clip, stream);
    default:
      return launchTyped<Real, RG_GRID_LENNARD_JONES_ATTRACTION, TRI>(p, ipos, ipar, bx, by, bz, count, clip, stream);
  }
}

// Launch geometry shared by every entry point: cell, spacing, pair cutoff, the brick's staging radii and the supercell
// clip. Returns whether the CLIP kernels are needed (the supercell that `cutoff` sizes is narrower than twice the pair
// cutoff along some axis).
bool setupGridParams(GridParams& gp, const rg::HostBox& box, const rg_forcefield* ff, double cutoff, int nx, int ny,
                     int nz, int bx, int by, int bz)
{
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) gp.cell[c][r] = box.c[c][r];
  gp.ncells[0] = static_cast<double>(nx - 1);
  gp.ncells[1] = static_cast<double>(ny - 1);
  gp.ncells[2] = static_cast<double>(nz - 1);
  for (int d = 0; d < 3; ++d) gp.delta[d] = 1.0 / gp.ncells[d];
  gp.nx = nx;
  gp.ny = ny;
  gp.nz = nz;
  const double rc = ff->cutoff_framework_vdw;
  gp.rc2 = rc * rc;
  double R = 0.0;  // brick half-diagonal
  for (int sx = -1; sx <= 1; sx += 2)
    for (int sy = -1; sy <= 1; sy += 2)
      for (int sz = -1; sz <= 1; sz += 2)
      {
        double f[3] = {sx * 0.5 * (bx - 1) * gp.delta[0], sy * 0.5 * (by - 1) * gp.delta[1],
                       sz * 0.5 * (bz - 1) * gp.delta[2]},
               d[3];
        rg::matvec(box.c, f, d);
        R = std::fmax(R, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
      }
  const double rf = rc + R + 1e-6;
  gp.filter2 = rf * rf;
  // near images: within kNearRadius + R of the brick centre, so that every pair closer than kNearRadius is among them
  const double rn = kNearRadius + R;
  gp.near2 = rn * rn;
  gp.alpha = ff->ewald_alpha;
  gp.coul = rg::coulombFactor();
  gp.overlap = ff->overlap_criteria;
  return rg::supercellClip(box, rc, cutoff, gp.clip_h, gp.clip_ic);
}

constexpr int kSlabs = 8;  // z-slabs of a grid whose host copy overlaps the build

// Launches the grid kernel in z-slabs of bricks when host copies are wanted: after each slab, that slab of every
// output grid (a contiguous range of the layout data[l + 8*(i + nx*(j + ny*k))]) is copied to its host buffer on the
// context's copy stream, so the copies run while the later slabs (and the next grids of a set) are computed. Without
// host outputs it is one launch. The caller joins the copy stream before synchronising.
template <typename Launch>
rg_status launchSlabbed(rg_ctx* ctx, GridParams& gp, int bz, double* const* dev, double* const* host, int n_out,
                        Launch launch)
{
  bool any = false;
  for (int q = 0; q < n_out; ++q) any = any || (host && host[q]);
  const int zb = (gp.nz + bz - 1) / bz;
  const int n_slabs = any ? std::min(zb, kSlabs) : 1;
  cudaStream_t cs = nullptr;
  if (any)
  {
    rg_status st = rg::copyStream(ctx, &cs);
    if (st) return st;
  }
  const size_t plane = 8 * static_cast<size_t>(gp.nx) * gp.ny;  // doubles per z-plane
  for (int sl = 0; sl < n_slabs; ++sl)
  {
    gp.zb0 = any ? sl * zb / n_slabs : 0;
    gp.zb1 = any ? (sl + 1) * zb / n_slabs : 0;
    cudaError_t err = launch(gp);
    if (err != cudaSuccess) return rg::cudaFail(ctx, err, "gridKernel launch");
    if (!any) continue;
    cudaEvent_t ev = nullptr;
    rg_status st = rg::event(ctx, 1 + sl, &ev);
    if (st) return st;
    RG_CUDA(ctx, cudaEventRecord(ev, ctx->stream));
    RG_CUDA(ctx, cudaStreamWaitEvent(cs, ev, 0));
    const size_t k0 = static_cast<size_t>(gp.zb0) * bz, k1 = std::min<size_t>(gp.nz, static_cast<size_t>(gp.zb1) * bz);
    for (int q = 0; q < n_out; ++q)
      if (host && host[q] && k1 > k0)
        RG_CUDA(ctx, cudaMemcpyAsync(host[q] + plane * k0, dev[q] + plane * k0, sizeof(double) * plane * (k1 - k0),
                                     cudaMemcpyDeviceToHost, cs));
  }
  gp.zb0 = gp.zb1 = 0;
  return RG_OK;
}

}  // namespace

namespace rg
{
// Periodic images of the unit-cell atoms that can lie within rc of some point of the closed unit cell.
// pos.w carries C*q for the Ewald grid; par = (4 eps, sigma^2, shift) for Lennard-Jones grids.
int buildGridImages(int grid_type, const rg_forcefield* ff, const HostBox& box, const rg_atom* atoms, int n,
                    int probe_type, std::vector<double4>& pos, std::vector<double4>& par)
{
  double w[3];
  perpendicularWidths(box, w);
  const double rc = ff->cutoff_framework_vdw;
  const double C = coulombFactor();
  pos.clear();
  par.clear();
  for (int a = 0; a < n; ++a)
  {
    const rg_atom& at = atoms[a];
    double4 pr = make_double4(0, 0, 0, 0);
    double wq = 0.0;
    if (grid_type == RG_GRID_EWALD_REAL)
    {
      if (at.charge == 0.0) continue;
      wq = C * at.charge;
    }
    else
    {
      int idx = probe_type * ff->n_types + at.type;
      double eps = ff->epsilon[idx];
      if (eps == 0.0) continue;
      pr = make_double4(4.0 * eps, ff->sigma[idx] * ff->sigma[idx], ff->shift[idx], 0.0);
    }
    double r[3] = {at.x, at.y, at.z}, s[3];
    matvec(box.ic, r, s);
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d)
    {
      double f = rc / w[d] + 1e-9;
      lo[d] = static_cast<int>(std::ceil(-s[d] - f));
      hi[d] = static_cast<int>(std::floor(1.0 - s[d] + f));
    }
    for (int mx = lo[0]; mx <= hi[0]; ++mx)
      for (int my = lo[1]; my <= hi[1]; ++my)
        for (int mz = lo[2]; mz <= hi[2]; ++mz)
        {
          double m[3] = {static_cast<double>(mx), static_cast<double>(my), static_cast<double>(mz)}, d[3];
          matvec(box.c, m, d);
          pos.push_back(make_double4(r[0] + d[0], r[1] + d[1], r[2] + d[2], wq));
          par.push_back(pr);
        }
  }
  return static_cast<int>(pos.size());
}
}  // namespace rg

namespace
{
// One grid; the host copy (if any) is queued on the copy stream slab by slab. sync_out: join the copies and wait.
rg_status buildOne(rg_ctx* ctx, int grid_type, const rg_forcefield* ff, const rg_box* unit_cell,
                   const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, double cutoff, int nx, int ny, int nz,
                   int precision, double* out_device, double* out_host, rg_grid_stats* stats, bool sync_out)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  if (!ff || !unit_cell || (n_unit_atoms > 0 && !unit_atoms) || n_unit_atoms < 0)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: null argument");
  if (grid_type < 0 || grid_type > 3) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: bad grid_type");
  if (precision != RG_PRECISION_FP64 && precision != RG_PRECISION_FP32C)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: bad precision");
  if (nx < 2 || ny < 2 || nz < 2) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: need >= 2 points per axis");
  if (grid_type != RG_GRID_EWALD_REAL && (probe_type < 0 || probe_type >= ff->n_types))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: probe_type out of range");
  if (!out_device && !out_host) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: no output");
  if (!(cutoff > 0.0)) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build: cutoff must be positive");
  if (rg_status fs = rg::checkFinite(ctx, unit_atoms, n_unit_atoms, "rg_grid_build")) return fs;
  if (rg_status fs = rg::checkFiniteBox(ctx, unit_cell, "rg_grid_build")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));

  rg::HostBox box = rg::makeHostBox(unit_cell);
  std::vector<double4> hpos, hpar;
  int n_images = rg::buildGridImages(grid_type, ff, box, unit_atoms, n_unit_atoms, probe_type, hpos, hpar);

  const size_t npts = static_cast<size_t>(nx) * ny * nz;
  const size_t out_bytes = npts * 8 * sizeof(double);
  double* dout = out_device;
  void* p = nullptr;
  if (!dout)
  {
    rg_status st = rg::scratch(ctx, 0, out_bytes, &p);
    if (st) return st;
    dout = static_cast<double*>(p);
  }
  // images + pair counter in scratch slot 1
  size_t img_bytes = 2 * sizeof(double4) * static_cast<size_t>(n_images > 0 ? n_images : 1);
  rg_status st = rg::scratch(ctx, 1, img_bytes + 64, &p);
  if (st) return st;
  double4* dpos = static_cast<double4*>(p);
  double4* dpar = dpos + (n_images > 0 ? n_images : 1);
  unsigned long long* dcount = reinterpret_cast<unsigned long long*>(dpar + (n_images > 0 ? n_images : 1));
  if (n_images > 0)
  {
    // stage through pinned memory so the upload is asynchronous on the context stream; the staging slot is reused by
    // the next call only after this stream has passed the copy
    void* hp = nullptr;
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    st = rg::pinnedScratch(ctx, 0, 2 * sizeof(double4) * n_images, &hp);
    if (st) return st;
    double4* stage = static_cast<double4*>(hp);
    std::memcpy(stage, hpos.data(), sizeof(double4) * n_images);
    std::memcpy(stage + n_images, hpar.data(), sizeof(double4) * n_images);
    RG_CUDA(ctx, cudaMemcpyAsync(dpos, stage, 2 * sizeof(double4) * n_images, cudaMemcpyHostToDevice, ctx->stream));
  }
  RG_CUDA(ctx, cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), ctx->stream));

  // brick shape, staging radii and supercell
  const int bx = 8, by = 8, bz = 4;
  GridParams gp{};
  const bool clip = setupGridParams(gp, box, ff, cutoff, nx, ny, nz, bx, by, bz);
  gp.n_images = n_images;
  gp.pair_count = dcount;
  gp.out[0] = dout;
  gp.out[1] = nullptr;

  const bool count = stats != nullptr;
  double* devs[1] = {dout};
  double* hosts[1] = {out_host};
  rg_status lst = launchSlabbed(ctx, gp, bz, devs, hosts, 1, [&](const GridParams& g) {
    if (precision == RG_PRECISION_FP64)
      return box.triclinic ? launchPrec<double, true>(grid_type, g, dpos, dpar, bx, by, bz, count, clip, ctx->stream)
                           : launchPrec<double, false>(grid_type, g, dpos, dpar, bx, by, bz, count, clip, ctx->stream);
    return box.triclinic ? launchPrec<float, true>(grid_type, g, dpos, dpar, bx, by, bz, count, clip, ctx->stream)
                         : launchPrec<float, false>(grid_type, g, dpos, dpar, bx, by, bz, count, clip, ctx->stream);
  });
  if (lst) return lst;
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
  if (out_host && sync_out)
  {
    rg_status st2 = rg::joinCopies(ctx);
    if (st2) return st2;
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return RG_OK;
}
}  // namespace

extern "C" rg_status rg_grid_build(rg_ctx* ctx, int grid_type, const rg_forcefield* ff, const rg_box* unit_cell,
                                   const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, double cutoff, int nx,
                                   int ny, int nz, int precision, double* out_device, double* out_host,
                                   rg_grid_stats* stats)
{
  return buildOne(ctx, grid_type, ff, unit_cell, unit_atoms, n_unit_atoms, probe_type, cutoff, nx, ny, nz, precision,
                  out_device, out_host, stats, true);
}

// ---------------------------------------------------------------------------------------------------------------------
// Grid build without any allocation by the library.
//
// For callers that cannot allocate device memory themselves or let a library do it: an application whose device
// memory is owned by another allocator (a host framework that reserves the whole device up front, or a pool with a
// hard budget), where an extra cudaMalloc would fail or break the budget. The caller passes the inputs and the device
// output; the only working memory is the file-scope array below, whose size is fixed at load time.
// ---------------------------------------------------------------------------------------------------------------------
namespace
{
// Scratch of the no-allocation grid build: up to kNoAllocMaxImages staged periodic images (position + parameters,
// 2 x 32 bytes each) followed by the 8-byte pair counter. Every GPU that loads this library holds it until exit.
constexpr int kNoAllocMaxImages = 32768;
constexpr size_t kNoAllocBytes = 2 * sizeof(double4) * kNoAllocMaxImages + 256;
__device__ __align__(256) unsigned char g_grid_noalloc_scratch[kNoAllocBytes];

// The device address of g_grid_noalloc_scratch on `device`, which must be current. Looked up on every call (a host-side
// query, no allocation) so that no address outlives the context it belongs to; in host code the symbol itself is only a
// host-side stand-in and must never be passed to a kernel.
cudaError_t noallocScratchAddress(void** out) { return cudaGetSymbolAddress(out, g_grid_noalloc_scratch); }
}  // namespace

namespace
{
// The body of rg_grid_build_noalloc, with `device` current.
rg_status gridBuildNoalloc(int device, cudaStream_t st, int grid_type, const rg_forcefield* ff, const rg_box* unit_cell,
                           const rg_atom* unit_atoms, int n_unit_atoms, int probe_type, double cutoff, int nx, int ny,
                           int nz, int precision, double* out_device, rg_grid_stats* stats)
{
  void* base = nullptr;
  if (noallocScratchAddress(&base) != cudaSuccess) return RG_ERR_CUDA;
  double4* dpos = static_cast<double4*>(base);
  double4* dpar = dpos + kNoAllocMaxImages;
  unsigned long long* dcount = reinterpret_cast<unsigned long long*>(dpar + kNoAllocMaxImages);

  const rg::HostBox box = rg::makeHostBox(unit_cell);
  double w[3];
  rg::perpendicularWidths(box, w);
  const double rc = ff->cutoff_framework_vdw;
  const double C = rg::coulombFactor();

  // Enumerate the images in the order of rg_grid_build and stream them to the scratch array through a fixed stack
  // buffer (copies from pageable memory return once the buffer may be reused). Sizes beyond the array are rejected.
  constexpr int kChunk = 256;
  double4 cpos[kChunk], cpar[kChunk];
  int in_chunk = 0, n_images = 0;
  bool too_many = false;
  auto flush = [&]() -> bool
  {
    if (in_chunk == 0) return true;
    if (cudaMemcpyAsync(dpos + n_images - in_chunk, cpos, sizeof(double4) * in_chunk, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(dpar + n_images - in_chunk, cpar, sizeof(double4) * in_chunk, cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
      return false;
    if (cudaStreamSynchronize(st) != cudaSuccess) return false;
    in_chunk = 0;
    return true;
  };
  for (int a = 0; a < n_unit_atoms && !too_many; ++a)
  {
    const rg_atom& at = unit_atoms[a];
    double4 pr = make_double4(0, 0, 0, 0);
    double wq = 0.0;
    if (grid_type == RG_GRID_EWALD_REAL)
    {
      if (at.charge == 0.0) continue;
      wq = C * at.charge;
    }
    else
    {
      const int idx = probe_type * ff->n_types + at.type;
      if (ff->epsilon[idx] == 0.0) continue;
      pr = make_double4(4.0 * ff->epsilon[idx], ff->sigma[idx] * ff->sigma[idx], ff->shift[idx], 0.0);
    }
    double r[3] = {at.x, at.y, at.z}, s[3];
    rg::matvec(box.ic, r, s);
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d)
    {
      const double f = rc / w[d] + 1e-9;
      lo[d] = static_cast<int>(std::ceil(-s[d] - f));
      hi[d] = static_cast<int>(std::floor(1.0 - s[d] + f));
    }
    for (int mx = lo[0]; mx <= hi[0] && !too_many; ++mx)
      for (int my = lo[1]; my <= hi[1] && !too_many; ++my)
        for (int mz = lo[2]; mz <= hi[2] && !too_many; ++mz)
        {
          if (n_images == kNoAllocMaxImages)
          {
            too_many = true;
            break;
          }
          double m[3] = {static_cast<double>(mx), static_cast<double>(my), static_cast<double>(mz)}, d[3];
          rg::matvec(box.c, m, d);
          cpos[in_chunk] = make_double4(r[0] + d[0], r[1] + d[1], r[2] + d[2], wq);
          cpar[in_chunk] = pr;
          ++in_chunk;
          ++n_images;
          if (in_chunk == kChunk && !flush()) return RG_ERR_CUDA;
        }
  }
  if (too_many) return RG_ERR_INVALID_ARGUMENT;  // more than kNoAllocMaxImages periodic images
  if (!flush()) return RG_ERR_CUDA;
  // the counter must start at zero; the array keeps whatever the previous call left
  if (cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st) != cudaSuccess) return RG_ERR_CUDA;

  const int bx = 8, by = 8, bz = 4;
  GridParams gp{};
  const bool clip = setupGridParams(gp, box, ff, cutoff, nx, ny, nz, bx, by, bz);
  gp.n_images = n_images;
  gp.pair_count = dcount;
  gp.out[0] = out_device;
  gp.out[1] = nullptr;
  const bool count = stats != nullptr;
  cudaError_t err;
  if (precision == RG_PRECISION_FP64)
    err = box.triclinic ? launchPrec<double, true>(grid_type, gp, dpos, dpar, bx, by, bz, count, clip, st)
                        : launchPrec<double, false>(grid_type, gp, dpos, dpar, bx, by, bz, count, clip, st);
  else
    err = box.triclinic ? launchPrec<float, true>(grid_type, gp, dpos, dpar, bx, by, bz, count, clip, st)
                        : launchPrec<float, false>(grid_type, gp, dpos, dpar, bx, by, bz, count, clip, st);
  if (err != cudaSuccess) return RG_ERR_CUDA;
  if (stats)
  {
    unsigned long long c = 0;
    if (cudaMemcpyAsync(&c, dcount, sizeof(c), cudaMemcpyDeviceToHost, st) != cudaSuccess) return RG_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return RG_ERR_CUDA;
    stats->pair_count = static_cast<int64_t>(c);
    stats->n_images = n_images;
    stats->h2d_bytes = static_cast<int64_t>(2 * sizeof(double4)) * n_images;
    stats->d2h_bytes = 0;
  }
  return RG_OK;
}
}  // namespace

extern "C" rg_status rg_grid_build_noalloc(int device, void* stream, int grid_type, const rg_forcefield* ff,
                                           const rg_box* unit_cell, const rg_atom* unit_atoms, int n_unit_atoms,
                                           int probe_type, double cutoff, int nx, int ny, int nz, int precision,
                                           double* out_device, rg_grid_stats* stats)
{
  if (!ff || !unit_cell || (n_unit_atoms > 0 && !unit_atoms) || n_unit_atoms < 0 || !out_device)
    return RG_ERR_INVALID_ARGUMENT;
  if (grid_type < 0 || grid_type > 3 || (precision != RG_PRECISION_FP64 && precision != RG_PRECISION_FP32C))
    return RG_ERR_INVALID_ARGUMENT;
  if (nx < 2 || ny < 2 || nz < 2 || !(cutoff > 0.0)) return RG_ERR_INVALID_ARGUMENT;
  if (rg_status fs = rg::checkFinite(nullptr, unit_atoms, n_unit_atoms, "rg_grid_build_noalloc")) return fs;
  if (rg_status fs = rg::checkFiniteBox(nullptr, unit_cell, "rg_grid_build_noalloc")) return fs;
  if (grid_type != RG_GRID_EWALD_REAL && (probe_type < 0 || probe_type >= ff->n_types)) return RG_ERR_INVALID_ARGUMENT;
  int n_devices = 0;
  if (cudaGetDeviceCount(&n_devices) != cudaSuccess) return RG_ERR_CUDA;
  if (device < 0 || device >= n_devices) return RG_ERR_INVALID_ARGUMENT;
  // the work runs with `device` current; the caller's current device is restored on every return
  int previous = -1;
  if (cudaGetDevice(&previous) != cudaSuccess) return RG_ERR_CUDA;
  if (previous != device && cudaSetDevice(device) != cudaSuccess) return RG_ERR_CUDA;
  const rg_status status = gridBuildNoalloc(device, static_cast<cudaStream_t>(stream), grid_type, ff, unit_cell,
                                            unit_atoms, n_unit_atoms, probe_type, cutoff, nx, ny, nz, precision,
                                            out_device, stats);
  if (previous != device && cudaSetDevice(previous) != cudaSuccess) return RG_ERR_CUDA;
  return status;
}

// ---------------------------------------------------------------------------------------------------------------------
// Several grids of one framework in one call: the loop of System::createFrameworkInterpolationGrids
// (src/raspakit/system_interpolation_grids.cpp:202-238). Lennard-Jones grids whose probes see the same framework atoms
// (nonzero epsilon for the same atoms) are built two at a time by one kernel that shares the candidate staging, the
// distances and the reciprocal between the two probes.
// ---------------------------------------------------------------------------------------------------------------------
extern "C" rg_status rg_grid_build_set(rg_ctx* ctx, const rg_forcefield* ff, const rg_box* unit_cell,
                                       const rg_atom* unit_atoms, int n_unit_atoms, double cutoff, int nx, int ny,
                                       int nz, int precision, int n_grids, const int* grid_types,
                                       const int* probe_types, double* const* out_device, double* const* out_host,
                                       rg_grid_stats* stats)
{
  if (!ctx) return RG_ERR_INVALID_ARGUMENT;
  if (!ff || !unit_cell || (n_unit_atoms > 0 && !unit_atoms) || n_unit_atoms < 0 || n_grids < 0 ||
      (n_grids > 0 && (!grid_types || !probe_types || !out_device)))
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: null argument");
  if (precision != RG_PRECISION_FP64 && precision != RG_PRECISION_FP32C)
    return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: bad precision");
  if (nx < 2 || ny < 2 || nz < 2) return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: grid shape");
  for (int g = 0; g < n_grids; ++g)
  {
    if (grid_types[g] < 0 || grid_types[g] > 3 || !out_device[g])
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: bad grid type or output");
    if (grid_types[g] != RG_GRID_EWALD_REAL && (probe_types[g] < 0 || probe_types[g] >= ff->n_types))
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: probe_type out of range");
  }
  // the cutoff that sizes each grid's supercell: the caller's, or the reference's per type (cutOffCoulomb for the Ewald
  // grid, cutOffFrameworkVDW for the VDW grids; system_interpolation_grids.cpp:211, 236)
  auto gridCutoff = [&](int type)
  { return cutoff > 0.0 ? cutoff : (type == RG_GRID_EWALD_REAL ? ff->cutoff_coulomb : ff->cutoff_framework_vdw); };
  for (int g = 0; g < n_grids; ++g)
    if (!(gridCutoff(grid_types[g]) > 0.0))
      return rg::fail(ctx, RG_ERR_INVALID_ARGUMENT, "rg_grid_build_set: cutoff must be positive");
  if (rg_status fs = rg::checkFinite(ctx, unit_atoms, n_unit_atoms, "rg_grid_build_set")) return fs;
  if (rg_status fs = rg::checkFiniteBox(ctx, unit_cell, "rg_grid_build_set")) return fs;
  RG_CUDA(ctx, cudaSetDevice(ctx->device));
  const rg::HostBox box = rg::makeHostBox(unit_cell);
  // which framework atoms a Lennard-Jones probe sees
  auto mask = [&](int probe)
  {
    std::vector<char> m(n_unit_atoms);
    for (int a = 0; a < n_unit_atoms; ++a) m[a] = ff->epsilon[probe * ff->n_types + unit_atoms[a].type] != 0.0;
    return m;
  };
  std::vector<int> done(n_grids, 0);
  const size_t grid_bytes = sizeof(double) * 8 * static_cast<size_t>(nx) * ny * nz;
  for (int g = 0; g < n_grids; ++g)
  {
    if (done[g]) continue;
    int partner = -1;
    if (grid_types[g] == RG_GRID_LENNARD_JONES)
    {
      const std::vector<char> mg = mask(probe_types[g]);
      for (int h = g + 1; h < n_grids && partner < 0; ++h)
        if (!done[h] && grid_types[h] == RG_GRID_LENNARD_JONES && mask(probe_types[h]) == mg) partner = h;
    }
    if (partner < 0)
    {
      rg_status st = buildOne(ctx, grid_types[g], ff, unit_cell, unit_atoms, n_unit_atoms, probe_types[g],
                              gridCutoff(grid_types[g]), nx, ny, nz, precision, out_device[g],
                              out_host ? out_host[g] : nullptr,
                              stats ? &stats[g] : nullptr, false);
      if (st) return st;
      done[g] = 1;
      continue;
    }
    // fused pair: positions from probe g, parameters of both probes interleaved per image
    std::vector<double4> pos, par0, pos1, par1;
    const int n_images = rg::buildGridImages(RG_GRID_LENNARD_JONES, ff, box, unit_atoms, n_unit_atoms,
                                             probe_types[g], pos, par0);
    rg::buildGridImages(RG_GRID_LENNARD_JONES, ff, box, unit_atoms, n_unit_atoms, probe_types[partner], pos1, par1);
    void* p = nullptr;
    const int nimg = n_images > 0 ? n_images : 1;
    rg_status st = rg::scratch(ctx, 1, 3 * sizeof(double4) * static_cast<size_t>(nimg) + 64, &p);
    if (st) return st;
    double4* dpos = static_cast<double4*>(p);
    double4* dpar = dpos + nimg;
    unsigned long long* dcount = reinterpret_cast<unsigned long long*>(dpar + 2 * static_cast<size_t>(nimg));
    if (n_images > 0)
    {
      void* hp = nullptr;
      RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      st = rg::pinnedScratch(ctx, 0, 3 * sizeof(double4) * n_images, &hp);
      if (st) return st;
      double4* stage = static_cast<double4*>(hp);
      std::memcpy(stage, pos.data(), sizeof(double4) * n_images);
      for (int i = 0; i < n_images; ++i)
      {
        stage[n_images + 2 * i] = par0[i];
        stage[n_images + 2 * i + 1] = par1[i];
      }
      RG_CUDA(ctx, cudaMemcpyAsync(dpos, stage, 3 * sizeof(double4) * n_images, cudaMemcpyHostToDevice, ctx->stream));
    }
    RG_CUDA(ctx, cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), ctx->stream));
    const int bx = 8, by = 8, bz = 4;
    GridParams gp{};
    const bool clip = setupGridParams(gp, box, ff, gridCutoff(RG_GRID_LENNARD_JONES), nx, ny, nz, bx, by, bz);
    gp.n_images = n_images;
    gp.pair_count = dcount;
    gp.out[0] = out_device[g];
    gp.out[1] = out_device[partner];
    const bool count = stats != nullptr;
    double* devs[2] = {out_device[g], out_device[partner]};
    double* hosts[2] = {out_host ? out_host[g] : nullptr, out_host ? out_host[partner] : nullptr};
    st = launchSlabbed(ctx, gp, bz, devs, hosts, 2, [&](const GridParams& q) {
      if (precision == RG_PRECISION_FP64)
        return box.triclinic ? launchTyped<double, RG_GRID_LENNARD_JONES, true, 2>(q, dpos, dpar, bx, by, bz, count,
                                                                                   clip, ctx->stream)
                             : launchTyped<double, RG_GRID_LENNARD_JONES, false, 2>(q, dpos, dpar, bx, by, bz, count,
                                                                                    clip, ctx->stream);
      return box.triclinic ? launchTyped<float, RG_GRID_LENNARD_JONES, true, 2>(q, dpos, dpar, bx, by, bz, count, clip,
                                                                                ctx->stream)
                           : launchTyped<float, RG_GRID_LENNARD_JONES, false, 2>(q, dpos, dpar, bx, by, bz, count, clip,
                                                                                 ctx->stream);
    });
    if (st) return st;
    if (stats)
    {
      unsigned long long c = 0;
      RG_CUDA(ctx, cudaMemcpyAsync(&c, dcount, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
      RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      for (int q : {g, partner})
      {
        stats[q].pair_count = static_cast<int64_t>(c);
        stats[q].n_images = n_images;
        stats[q].h2d_bytes = static_cast<int64_t>(3 * sizeof(double4)) * n_images / 2;
        stats[q].d2h_bytes = (out_host && out_host[q]) ? static_cast<int64_t>(grid_bytes) : 0;
      }
    }
    done[g] = done[partner] = 1;
  }
  if (out_host)
  {
    rg_status st = rg::joinCopies(ctx);
    if (st) return st;
    RG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return RG_OK;
}

// Device-side pair potentials, periodic boundaries and tricubic grid interpolation shared by the CBMC trial-energy
// kernels and the device-resident Monte Carlo kernels. All FP64.
#pragma once

#include <cuda_runtime.h>

#include "../../include/raspa_gpu.h"

namespace rgd
{
// Force-field tables on the device (n x n, row = type A).
struct FF
{
  int n;
  const double* eps4;   // 4 * epsilon
  const double* sig2;   // sigma^2
  const double* shift;
  const int* lj;
  double alpha;
  double coul;          // CoulombicConversionFactor
  double overlap;
  int use_charge;
};

struct Box
{
  double c[3][3];   // c[col][row]
  double ic[3][3];
  int triclinic;
  double volume;
};

__device__ __forceinline__ double roundHalfAway(double x)
{
  return static_cast<double>(static_cast<long long>(x + ((x >= 0.0) ? 0.5 : -0.5)));
}

// SimulationBox::applyPeriodicBoundaryConditions (src/raspakit/simulationbox.ixx:131-161)
__device__ __forceinline__ void pbc(const Box& b, double& dx, double& dy, double& dz)
{
  if (!b.triclinic)
  {
    dx -= roundHalfAway(dx * b.ic[0][0]) * b.c[0][0];
    dy -= roundHalfAway(dy * b.ic[1][1]) * b.c[1][1];
    dz -= roundHalfAway(dz * b.ic[2][2]) * b.c[2][2];
    return;
  }
  double s0 = b.ic[0][0] * dx + b.ic[1][0] * dy + b.ic[2][0] * dz;
  double s1 = b.ic[0][1] * dx + b.ic[1][1] * dy + b.ic[2][1] * dz;
  double s2 = b.ic[0][2] * dx + b.ic[1][2] * dy + b.ic[2][2] * dz;
  s0 -= roundHalfAway(s0);
  s1 -= roundHalfAway(s1);
  s2 -= roundHalfAway(s2);
  dx = b.c[0][0] * s0 + b.c[1][0] * s1 + b.c[2][0] * s2;
  dy = b.c[0][1] * s0 + b.c[1][1] * s1 + b.c[2][1] * s2;
  dz = b.c[0][2] * s0 + b.c[1][2] * s1 + b.c[2][2] * s2;
}

// potentialVDW<0>, Lennard-Jones branch (src/raspakit/potentials/pair_vdw.ixx:85-101): {energy, dU/dlambda}
__device__ __forceinline__ double2 pairVDW(const FF& ff, double sA, double sB, double rr, int tA, int tB)
{
  const int idx = tA * ff.n + tB;
  if (!ff.lj[idx]) return make_double2(0.0, 0.0);
  const double scaling = sA * sB;
  const double arg1 = ff.eps4[idx];
  const double arg2 = ff.sig2[idx];
  const double arg3 = ff.shift[idx];
  const double temp = rr / arg2;
  const double temp3 = temp * temp * temp;
  const double inv_scaling = 1.0 - scaling;
  const double rri3 = 1.0 / (temp3 + 0.5 * inv_scaling * inv_scaling);
  const double rri6 = rri3 * rri3;
  const double term = arg1 * (rri3 * (rri3 - 1.0)) - arg3;
  const double dlambda_term = arg1 * scaling * inv_scaling * (2.0 * rri6 * rri3 - rri6);
  return make_double2(scaling * term, term + dlambda_term);
}

// potentialCoulomb<0>, Ewald branch (src/raspakit/potentials/pair_coulomb.ixx:51-77): {energy, dU/dlambda}
__device__ __forceinline__ double2 pairCoulomb(const FF& ff, double sA, double sB, double r, double qA, double qB)
{
  const double scaling = sA * sB;
  const double alpha = ff.alpha;
  const double prefactor = ff.coul * qA * qB;
  const double s = r + 0.01 * (1.0 - scaling);
  const double inverseS = 1.0 / s;
  const double inverseSS = inverseS * inverseS;
  const double erfcTerm = erfc(alpha * s);
  const double gaussian = exp(-alpha * alpha * s * s) * 0.564189583547756286948079451560772586;
  const double phi = erfcTerm * inverseS;
  const double phiPrime = -(erfcTerm * inverseSS + 2.0 * alpha * gaussian * inverseS);
  return make_double2(scaling * prefactor * phi, prefactor * (phi - scaling * 0.01 * phiPrime));
}

struct Grid
{
  const double* data;  // 8 doubles per point, data[l + 8*(i + nx*(j + ny*k))]
  int nx, ny, nz;
  double ic[3][3];     // inverse of the grid's unit cell
};

__device__ __forceinline__ double fract1(double x)
{
  // double3::fract (src/mathkit/double3.cpp:22-50)
  double s = x - rint(x);
  if (s < 0.0) s += 1.0;
  if (s > 1.0) s -= 1.0;
  return s;
}

// InterpolationEnergyGrid::interpolate, tricubic scheme (src/raspakit/interpolation_energy_grid.cpp:3980-4118).
// The reference maps the 64 corner values (f, fx, fy, fz, fxy, fxz, fyz, fxyz at 8 corners) through the Lekien-Marsden
// 64x64 matrix to monomial coefficients and sums the polynomial; that interpolant is the tensor product of 1D cubic
// Hermite bases, evaluated here directly as 64 products (identical up to rounding).
// The grid cell of a position and the 1D cubic Hermite bases of its local coordinates.
struct GridCell
{
  int i0[3];
  double h[3][2][2];  // h[d][corner][order]: corner 0/1, order 0 = value basis, 1 = derivative basis
};

__device__ __forceinline__ GridCell gridCell(const Grid& g, double px, double py, double pz)
{
  GridCell cl;
  double s[3];
  s[0] = fract1(g.ic[0][0] * px + g.ic[1][0] * py + g.ic[2][0] * pz);
  s[1] = fract1(g.ic[0][1] * px + g.ic[1][1] * py + g.ic[2][1] * pz);
  s[2] = fract1(g.ic[0][2] * px + g.ic[1][2] * py + g.ic[2][2] * pz);
  const int nc[3] = {g.nx - 1, g.ny - 1, g.nz - 1};
  double t[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    long long c = static_cast<long long>(s[d] * static_cast<double>(nc[d]));
    cl.i0[d] = static_cast<int>(c < nc[d] - 1 ? c : nc[d] - 1);
    t[d] = s[d] * static_cast<double>(nc[d]) - static_cast<double>(cl.i0[d]);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const double x = t[d], x2 = x * x, x3 = x2 * x;
    cl.h[d][0][0] = 2.0 * x3 - 3.0 * x2 + 1.0;
    cl.h[d][1][0] = -2.0 * x3 + 3.0 * x2;
    cl.h[d][0][1] = x3 - 2.0 * x2 + x;
    cl.h[d][1][1] = x3 - x2;
  }
  return cl;
}

// The share of one corner (0..7: bit 0 = x, 1 = y, 2 = z) of the cell: its 8 stored channels (f, fx, fy, fz, fxy,
// fxz, fyz, fxyz) times their basis products.
__device__ __forceinline__ double interpolateCorner(const Grid& g, const GridCell& cl, int corner)
{
  const int ox[8] = {0, 1, 0, 0, 1, 1, 0, 1};
  const int oy[8] = {0, 0, 1, 0, 1, 0, 1, 1};
  const int oz[8] = {0, 0, 0, 1, 0, 1, 1, 1};
  const int cx = corner & 1, cy = (corner >> 1) & 1, cz = (corner >> 2) & 1;
  const double* p = g.data + 8 * (static_cast<long long>(cl.i0[0] + cx) +
                                  static_cast<long long>(g.nx) * (static_cast<long long>(cl.i0[1] + cy) +
                                                                 static_cast<long long>(g.ny) * (cl.i0[2] + cz)));
  const double2* p2 = reinterpret_cast<const double2*>(p);
  double v[8];
#pragma unroll
  for (int q = 0; q < 4; ++q)
  {
    double2 u = __ldg(p2 + q);
    v[2 * q] = u.x;
    v[2 * q + 1] = u.y;
  }
  double value = 0.0;
#pragma unroll
  for (int l = 0; l < 8; ++l) value += v[l] * cl.h[0][cx][ox[l]] * cl.h[1][cy][oy[l]] * cl.h[2][cz][oz[l]];
  return value;
}

// Value and Cartesian gradient of the interpolant (InterpolationEnergyGrid::interpolateHessian, tricubic branch,
// interpolation_energy_grid.cpp:4518-4590): the same tensor-product Hermite form, differentiated along each local cell
// coordinate t = s * (n - 1) - i0, then dE/ds = (n - 1) dE/dt and dE/dr_a = sum_b dE/ds_b * ic[a][b].
__device__ __forceinline__ double interpolateGradient(const Grid& g, double px, double py, double pz, double grad[3])
{
  const GridCell cl = gridCell(g, px, py, pz);
  double s[3];
  s[0] = fract1(g.ic[0][0] * px + g.ic[1][0] * py + g.ic[2][0] * pz);
  s[1] = fract1(g.ic[0][1] * px + g.ic[1][1] * py + g.ic[2][1] * pz);
  s[2] = fract1(g.ic[0][2] * px + g.ic[1][2] * py + g.ic[2][2] * pz);
  const int nc[3] = {g.nx - 1, g.ny - 1, g.nz - 1};
  double dh[3][2][2];  // d/dt of the bases
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const double t = s[d] * static_cast<double>(nc[d]) - static_cast<double>(cl.i0[d]), t2 = t * t;
    dh[d][0][0] = 6.0 * t2 - 6.0 * t;
    dh[d][1][0] = -6.0 * t2 + 6.0 * t;
    dh[d][0][1] = 3.0 * t2 - 4.0 * t + 1.0;
    dh[d][1][1] = 3.0 * t2 - 2.0 * t;
  }
  const int ox[8] = {0, 1, 0, 0, 1, 1, 0, 1};
  const int oy[8] = {0, 0, 1, 0, 1, 0, 1, 1};
  const int oz[8] = {0, 0, 0, 1, 0, 1, 1, 1};
  double value = 0.0, dt[3] = {0.0, 0.0, 0.0};
  for (int corner = 0; corner < 8; ++corner)
  {
    const int cx = corner & 1, cy = (corner >> 1) & 1, cz = (corner >> 2) & 1;
    const double* p = g.data + 8 * (static_cast<long long>(cl.i0[0] + cx) +
                                    static_cast<long long>(g.nx) * (static_cast<long long>(cl.i0[1] + cy) +
                                                                   static_cast<long long>(g.ny) * (cl.i0[2] + cz)));
#pragma unroll
    for (int l = 0; l < 8; ++l)
    {
      const double v = p[l];
      const double hx = cl.h[0][cx][ox[l]], hy = cl.h[1][cy][oy[l]], hz = cl.h[2][cz][oz[l]];
      value += v * hx * hy * hz;
      dt[0] += v * dh[0][cx][ox[l]] * hy * hz;
      dt[1] += v * hx * dh[1][cy][oy[l]] * hz;
      dt[2] += v * hx * hy * dh[2][cz][oz[l]];
    }
  }
  const double ds[3] = {dt[0] * nc[0], dt[1] * nc[1], dt[2] * nc[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) grad[a] = g.ic[a][0] * ds[0] + g.ic[a][1] * ds[1] + g.ic[a][2] * ds[2];
  return value;
}

__device__ __forceinline__ double interpolate(const Grid& g, double px, double py, double pz)
{
  const GridCell cl = gridCell(g, px, py, pz);
  double value = 0.0;
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) value += interpolateCorner(g, cl, corner);
  return value;
}

// Triquintic scheme (27 values per point, data[l + 27*(i + nx*(j + ny*k))]): channel l holds the mixed derivative of
// orders quinticOrder(l, axis) along the three cell axes, in units of the grid cell (makeFrameworkInterpolationGrid,
// interpolation_energy_grid.cpp:3882-3962). The reference maps the 216 corner values through a 216x216 matrix to the
// monomial coefficients of a polynomial of degree 5 per axis (computeCoefficients, :2116-3500); that polynomial is
// the tensor product of the 1D quintic Hermite bases (value, first and second derivative at both ends), evaluated
// here directly as 27 x 8 products.
__host__ __device__ constexpr int quinticOrder(int l, int axis)
{
  // orders (x, y, z) packed one per hex digit, x lowest
  constexpr int packed[27] = {0x000, 0x001, 0x010, 0x100, 0x002, 0x011, 0x101, 0x020, 0x110,
                              0x200, 0x012, 0x102, 0x021, 0x111, 0x120, 0x201, 0x210, 0x022,
                              0x202, 0x220, 0x112, 0x121, 0x211, 0x122, 0x212, 0x221, 0x222};
  return (packed[l] >> (4 * axis)) & 0xf;
}

// quintic Hermite bases of the corner at t = 0 (value, first, second derivative) and their derivatives; the corner at
// t = 1 uses u = 1 - t with the first-derivative basis negated
__device__ __forceinline__ void quinticBases(double t, double b[3], double db[3])
{
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  b[0] = 1.0 - 10.0 * t3 + 15.0 * t4 - 6.0 * t5;
  b[1] = t - 6.0 * t3 + 8.0 * t4 - 3.0 * t5;
  b[2] = 0.5 * t2 - 1.5 * t3 + 1.5 * t4 - 0.5 * t5;
  db[0] = -30.0 * t2 + 60.0 * t3 - 30.0 * t4;
  db[1] = 1.0 - 18.0 * t2 + 32.0 * t3 - 15.0 * t4;
  db[2] = t - 4.5 * t2 + 6.0 * t3 - 2.5 * t4;
}

// Value of the triquintic interpolant at a Cartesian position (InterpolationEnergyGrid::interpolate, triquintic
// branch, interpolation_energy_grid.cpp:4119-4178) and, if grad != nullptr, its Cartesian gradient
// (interpolateGradient, :4348-4410): dE/dt along each cell axis, times (n - 1), mapped with the inverse cell.
__device__ __forceinline__ double interpolateQuintic(const Grid& g, double px, double py, double pz, double* grad)
{
  double s[3];
  s[0] = fract1(g.ic[0][0] * px + g.ic[1][0] * py + g.ic[2][0] * pz);
  s[1] = fract1(g.ic[0][1] * px + g.ic[1][1] * py + g.ic[2][1] * pz);
  s[2] = fract1(g.ic[0][2] * px + g.ic[1][2] * py + g.ic[2][2] * pz);
  const int nc[3] = {g.nx - 1, g.ny - 1, g.nz - 1};
  int i0[3];
  // h[d][corner][order], dh = d/dt
  double h[3][2][3], dh[3][2][3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const long long c = static_cast<long long>(s[d] * static_cast<double>(nc[d]));
    i0[d] = static_cast<int>(c < nc[d] - 1 ? c : nc[d] - 1);
    const double t = s[d] * static_cast<double>(nc[d]) - static_cast<double>(i0[d]);
    double b[3], db[3];
    quinticBases(t, b, db);
#pragma unroll
    for (int o = 0; o < 3; ++o)
    {
      h[d][0][o] = b[o];
      dh[d][0][o] = db[o];
    }
    quinticBases(1.0 - t, b, db);
    h[d][1][0] = b[0];
    h[d][1][1] = -b[1];
    h[d][1][2] = b[2];
    dh[d][1][0] = -db[0];
    dh[d][1][1] = db[1];
    dh[d][1][2] = -db[2];
  }
  double value = 0.0, dt[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int corner = 0; corner < 8; ++corner)
  {
    const int cx = corner & 1, cy = (corner >> 1) & 1, cz = (corner >> 2) & 1;
    const double* p = g.data + 27 * (static_cast<long long>(i0[0] + cx) +
                                     static_cast<long long>(g.nx) * (static_cast<long long>(i0[1] + cy) +
                                                                    static_cast<long long>(g.ny) * (i0[2] + cz)));
#pragma unroll
    for (int l = 0; l < 27; ++l)
    {
      const double v = __ldg(p + l);
      const int ox = quinticOrder(l, 0), oy = quinticOrder(l, 1), oz = quinticOrder(l, 2);
      const double hx = h[0][cx][ox], hy = h[1][cy][oy], hz = h[2][cz][oz];
      value += v * hx * hy * hz;
      if (grad)
      {
        dt[0] += v * dh[0][cx][ox] * hy * hz;
        dt[1] += v * hx * dh[1][cy][oy] * hz;
        dt[2] += v * hx * hy * dh[2][cz][oz];
      }
    }
  }
  if (grad)
  {
    const double ds[3] = {dt[0] * nc[0], dt[1] * nc[1], dt[2] * nc[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) grad[a] = g.ic[a][0] * ds[0] + g.ic[a][1] * ds[1] + g.ic[a][2] * ds[2];
  }
  return value;
}

// second derivatives of the quintic Hermite bases of the corner at t = 0
__device__ __forceinline__ void quinticBases2(double t, double d2[3])
{
  const double t2 = t * t, t3 = t2 * t;
  d2[0] = -60.0 * t + 180.0 * t2 - 120.0 * t3;
  d2[1] = -36.0 * t + 96.0 * t2 - 60.0 * t3;
  d2[2] = 1.0 - 9.0 * t + 18.0 * t2 - 10.0 * t3;
}

// Value, Cartesian gradient and Hessian (xx, xy, xz, yy, yz, zz) of the triquintic interpolant
// (InterpolationEnergyGrid::interpolateHessian, triquintic branch, interpolation_energy_grid.cpp:4602-4748): the
// derivatives along the cell axes of the tensor-product Hermite form, times (n - 1) per axis, mapped with the inverse
// cell (grad = M^T g, H = M^T Hs M).
__device__ __forceinline__ double interpolateQuinticHessian(const Grid& g, double px, double py, double pz,
                                                            double grad[3], double hess[6])
{
  double s[3];
  s[0] = fract1(g.ic[0][0] * px + g.ic[1][0] * py + g.ic[2][0] * pz);
  s[1] = fract1(g.ic[0][1] * px + g.ic[1][1] * py + g.ic[2][1] * pz);
  s[2] = fract1(g.ic[0][2] * px + g.ic[1][2] * py + g.ic[2][2] * pz);
  const int nc[3] = {g.nx - 1, g.ny - 1, g.nz - 1};
  int i0[3];
  double h[3][2][3], dh[3][2][3], d2h[3][2][3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const long long c = static_cast<long long>(s[d] * static_cast<double>(nc[d]));
    i0[d] = static_cast<int>(c < nc[d] - 1 ? c : nc[d] - 1);
    const double t = s[d] * static_cast<double>(nc[d]) - static_cast<double>(i0[d]);
    double b[3], db[3], b2[3];
    quinticBases(t, b, db);
    quinticBases2(t, b2);
#pragma unroll
    for (int o = 0; o < 3; ++o)
    {
      h[d][0][o] = b[o];
      dh[d][0][o] = db[o];
      d2h[d][0][o] = b2[o];
    }
    quinticBases(1.0 - t, b, db);
    quinticBases2(1.0 - t, b2);
    h[d][1][0] = b[0];
    h[d][1][1] = -b[1];
    h[d][1][2] = b[2];
    dh[d][1][0] = -db[0];
    dh[d][1][1] = db[1];
    dh[d][1][2] = -db[2];
    d2h[d][1][0] = b2[0];
    d2h[d][1][1] = -b2[1];
    d2h[d][1][2] = b2[2];
  }
  double value = 0.0, dt[3] = {0.0, 0.0, 0.0}, ht[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int corner = 0; corner < 8; ++corner)
  {
    const int cx = corner & 1, cy = (corner >> 1) & 1, cz = (corner >> 2) & 1;
    const double* p = g.data + 27 * (static_cast<long long>(i0[0] + cx) +
                                     static_cast<long long>(g.nx) * (static_cast<long long>(i0[1] + cy) +
                                                                    static_cast<long long>(g.ny) * (i0[2] + cz)));
#pragma unroll
    for (int l = 0; l < 27; ++l)
    {
      const double v = __ldg(p + l);
      const int ox = quinticOrder(l, 0), oy = quinticOrder(l, 1), oz = quinticOrder(l, 2);
      const double hx = h[0][cx][ox], hy = h[1][cy][oy], hz = h[2][cz][oz];
      const double gx = dh[0][cx][ox], gy = dh[1][cy][oy], gz = dh[2][cz][oz];
      value += v * hx * hy * hz;
      dt[0] += v * gx * hy * hz;
      dt[1] += v * hx * gy * hz;
      dt[2] += v * hx * hy * gz;
      ht[0] += v * d2h[0][cx][ox] * hy * hz;
      ht[1] += v * gx * gy * hz;
      ht[2] += v * gx * hy * gz;
      ht[3] += v * hx * d2h[1][cy][oy] * hz;
      ht[4] += v * hx * gy * gz;
      ht[5] += v * hx * hy * d2h[2][cz][oz];
    }
  }
  const double gs[3] = {dt[0] * nc[0], dt[1] * nc[1], dt[2] * nc[2]};
  const double Hs[3][3] = {{ht[0] * nc[0] * nc[0], ht[1] * nc[0] * nc[1], ht[2] * nc[0] * nc[2]},
                           {ht[1] * nc[0] * nc[1], ht[3] * nc[1] * nc[1], ht[4] * nc[1] * nc[2]},
                           {ht[2] * nc[0] * nc[2], ht[4] * nc[1] * nc[2], ht[5] * nc[2] * nc[2]}};
#pragma unroll
  for (int a = 0; a < 3; ++a) grad[a] = g.ic[a][0] * gs[0] + g.ic[a][1] * gs[1] + g.ic[a][2] * gs[2];
  constexpr int pi[6] = {0, 0, 0, 1, 1, 2}, pj[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int q = 0; q < 6; ++q)
  {
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) acc += g.ic[pi[q]][a] * g.ic[pj[q]][b] * Hs[a][b];
    hess[q] = acc;
  }
  return value;
}

// Internal accessors between translation units: the device data of a system and of an Ewald state.
rg_status systemExport(rg_system* s, FF* ff, Box* box, const double** type_grids /*[64]*/, const double** ewald_grid,
                       int* n_types, int gdims[3], double gic[3][3], rg_ctx** ctx);
// the framework atoms of a system (device rg_atom array, count)
rg_status systemFramework(rg_system* s, const rg_atom** fw, int* n_fw);
// the interpolation scheme of a system's grids (RG_SCHEME_TRICUBIC or RG_SCHEME_TRIQUINTIC)
int systemScheme(const rg_system* s);
rg_status proposalExport(rg_proposal* p, const double** cdf, const double** density, int* G, double* eps);
rg_status ewaldExport(rg_ewald* e, const char4** kvec, const double** temp, const double2** s_rigid, int64_t* nk,
                      int kmax[3], double* alpha, double* single_ion_sum);

// The supercell's minimum image keeps a displacement iff it lies in (-1/2, 1/2] of the supercell along every axis
// (SimulationBox::applyPeriodicBoundaryConditions, simulationbox.ixx:131-161, in the supercell of
// makeFrameworkInterpolationGrid, interpolation_energy_grid.cpp:3812-3815).
template <bool TRICLINIC, typename R>
__device__ __forceinline__ bool insideSupercell(const R (&h)[3], const R (&ic)[9], R dx, R dy, R dz)
{
  if constexpr (!TRICLINIC)
    return dx > -h[0] && dx <= h[0] && dy > -h[1] && dy <= h[1] && dz > -h[2] && dz <= h[2];
  else
  {
    bool in = true;
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      const R sd = ic[3 * d] * dx + ic[3 * d + 1] * dy + ic[3 * d + 2] * dz;
      in = in && sd > R(-0.5) && sd <= R(0.5);
    }
    return in;
  }
}

__device__ __forceinline__ int groupOf(const rg_atom& a) { return a.group_fractional & 0x0f; }
__device__ __forceinline__ bool fractionalOf(const rg_atom& a) { return (a.group_fractional >> 4) != 0; }
}  // namespace rgd

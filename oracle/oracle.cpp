// FP64 CPU oracle for the RASPA3 energy paths — TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Each function restates the cited reference function in double precision, keeping its loop structure,
// its edge semantics (rr = max(0.1, rr), overlap clamps, duplicate periodic end-points, fractional derivative
// scaling, supercell minimum image) and its expression order where that order is visible in the source.
// Citations are file:line within the RASPA3 tree (src/raspakit/...).

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kInvSqrtPi = 0.564189583547756286948079451560772586;

// ---- units.cpp:14-98 (base constants from foundationkit/units.ixx:29-55) ----
constexpr double kAngstrom = 1e-10;
constexpr double kPicoSecond = 1e-12;
constexpr double kAtomicMassUnit = 1.6605402e-27;
constexpr double kElectronicChargeUnit = 1.60217733e-19;
constexpr double kMolarGasConstant = 8.314464919;
constexpr double kAvogadroConstant = 6.0221419947e23;
constexpr double kDielectricConstantVacuum = 8.8541878176e-12;

double energyConversionFactor()
{
  return kAtomicMassUnit * kAngstrom * kAngstrom / (kPicoSecond * kPicoSecond);
}
double coulombFactor()
{
  return kElectronicChargeUnit * kElectronicChargeUnit /
         (4.0 * kPi * kDielectricConstantVacuum * kAngstrom * energyConversionFactor());
}

// ---- boxes: SimulationBox (simulationbox.ixx:131-161, simulationbox.cpp:120-156) ----
struct Box
{
  double c[3][3];   // c[col][row]; column col is lattice vector col
  double ic[3][3];  // inverse, same convention
  bool triclinic;
  double volume;
};

void invert(const double m[3][3], double inv[3][3], double* det_out)
{
  // double3x3::inverse (mathkit/double3x3.cpp:102-118); mRC = row R, column C = m[C-1][R-1].
  double m11 = m[0][0], m12 = m[1][0], m13 = m[2][0];
  double m21 = m[0][1], m22 = m[1][1], m23 = m[2][1];
  double m31 = m[0][2], m32 = m[1][2], m33 = m[2][2];
  double det = m11 * (m22 * m33 - m23 * m32) - m12 * (m21 * m33 - m23 * m31) + m13 * (m21 * m32 - m22 * m31);
  inv[0][0] = (m22 * m33 - m32 * m23) / det;
  inv[0][1] = -(m21 * m33 - m31 * m23) / det;
  inv[0][2] = (m21 * m32 - m31 * m22) / det;
  inv[1][0] = -(m12 * m33 - m32 * m13) / det;
  inv[1][1] = (m11 * m33 - m31 * m13) / det;
  inv[1][2] = -(m11 * m32 - m31 * m12) / det;
  inv[2][0] = (m12 * m23 - m22 * m13) / det;
  inv[2][1] = -(m11 * m23 - m21 * m13) / det;
  inv[2][2] = (m11 * m22 - m21 * m12) / det;
  if (det_out) *det_out = det;
}

Box makeBox(const obox* b)
{
  Box box{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) box.c[c][r] = b->cell[3 * c + r];
  double det;
  invert(box.c, box.ic, &det);
  box.volume = det;
  box.triclinic = b->triclinic != 0;
  return box;
}

Box scaledBox(const Box& b, int nx, int ny, int nz)
{
  obox o{};
  int n[3] = {nx, ny, nz};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.cell[3 * c + r] = b.c[c][r] * static_cast<double>(n[c]);
  o.triclinic = b.triclinic ? 1 : 0;
  return makeBox(&o);
}

inline void matvec(const double m[3][3], const double v[3], double out[3])
{
  for (int r = 0; r < 3; ++r) out[r] = m[0][r] * v[0] + m[1][r] * v[1] + m[2][r] * v[2];
}

inline double roundHalfAway(double x) { return static_cast<double>(static_cast<long long>(x + ((x >= 0.0) ? 0.5 : -0.5))); }

// SimulationBox::applyPeriodicBoundaryConditions (simulationbox.ixx:131-161)
inline void pbc(const Box& b, double dr[3])
{
  if (!b.triclinic)
  {
    dr[0] = dr[0] - roundHalfAway(dr[0] * b.ic[0][0]) * b.c[0][0];
    dr[1] = dr[1] - roundHalfAway(dr[1] * b.ic[1][1]) * b.c[1][1];
    dr[2] = dr[2] - roundHalfAway(dr[2] * b.ic[2][2]) * b.c[2][2];
    return;
  }
  double s[3];
  matvec(b.ic, dr, s);
  for (int d = 0; d < 3; ++d) s[d] -= roundHalfAway(s[d]);
  matvec(b.c, s, dr);
}

// SimulationBox::perpendicularWidths (simulationbox.cpp:137-148)
void perpendicularWidths(const Box& b, double w[3])
{
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

// double3::fract (mathkit/double3.cpp:22-50)
inline double fract1(double x)
{
  double s = x - std::rint(x);
  if (s < 0.0) s += 1.0;
  if (s > 1.0) s -= 1.0;
  return s;
}

struct Factor
{
  double e, f1, f2, f3;
};

// potentialLennardJonesTricubicDerivative (potentials/interpolation/tricubic_derivative_lj.ixx:33-46) and the
// repulsion/attraction variants (:48-78).
inline Factor ljTricubic(int kind, double eps, double sigma, double shift, double r2)
{
  double arg1 = 4.0 * eps;
  double arg2 = sigma * sigma;
  double temp3 = (arg2 / r2) * (arg2 / r2) * (arg2 / r2);
  double r4 = r2 * r2;
  double r6 = r4 * r2;
  switch (kind)
  {
    case 2:
      return {arg1 * temp3 * temp3 - 0.0, -12.0 * arg1 * temp3 * temp3 / r2, 168.0 * arg1 * temp3 * temp3 / r4,
              -2688.0 * arg1 * temp3 * temp3 / r6};
    case 3:
      return {arg1 * temp3 - 0.0, -6.0 * arg1 * temp3 / r2, 48.0 * arg1 * temp3 / r4, -480.0 * arg1 * temp3 / r6};
    default:
      return {arg1 * (temp3 * temp3 - temp3) - shift, -6.0 * arg1 * (2.0 * temp3 * temp3 - temp3) / r2,
              24.0 * arg1 * (7.0 * temp3 * temp3 - 2.0 * temp3) / r4,
              -96.0 * arg1 * (28.0 * temp3 * temp3 - 5.0 * temp3) / r6};
  }
}

// potentialRealEwaldTricubicDerivative (potentials/interpolation/tricubic_derivative_real_ewald.ixx:32-56)
inline Factor ewaldTricubic(double alpha, double rr, double r, double qa, double qb)
{
  const double C = coulombFactor();
  double exp_factor = std::erfc(alpha * r);
  double temp = C * qa * qb * exp_factor / r;
  double exp_term_rr = 2.0 * alpha * r * std::exp(-alpha * alpha * rr) * kInvSqrtPi;
  double alpha_r = alpha * r;
  double alpha_r_2 = alpha_r * alpha_r;
  double alpha_r_4 = alpha_r_2 * alpha_r_2;
  double r3 = rr * r;
  double r5 = r3 * rr;
  double r7 = r5 * rr;
  return {temp, -C * qa * qb * ((exp_term_rr + exp_factor) / r3),
          C * qa * qb * ((exp_term_rr * (2.0 * alpha_r_2 + 3.0) + 3.0 * exp_factor) / r5),
          -C * qa * qb * ((exp_term_rr * (4.0 * alpha_r_4 + 10 * alpha_r_2 + 15.0) + 15.0 * exp_factor) / r7)};
}

inline Factor gridFactor(int grid_type, const off* ff, double rr, int typeA, const oatom& b)
{
  int n = ff->n_types;
  int idx = typeA * n + b.type;
  if (grid_type == 1) return ewaldTricubic(ff->ewald_alpha, rr, std::sqrt(rr), 1.0, b.charge);
  return ljTricubic(grid_type, ff->epsilon[idx], ff->sigma[idx], ff->shift[idx], rr);
}

// Interactions::calculateTricubicDerivativeAtPosition (interactions/framework_molecule_grid.cpp:76-144):
// Cartesian energy, gradient, Hessian and third-derivative tensor.
void tricubicCartesian(int grid_type, const off* ff, const Box& superBox, const double* posA, int typeA,
                       const oatom* atoms, int n, double& energy, double g[3], double h[3][3], double t[3][3][3])
{
  const double rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  energy = 0.0;
  std::memset(g, 0, 3 * sizeof(double));
  std::memset(h, 0, 9 * sizeof(double));
  std::memset(t, 0, 27 * sizeof(double));
  for (int a = 0; a < n; ++a)
  {
    double dr[3] = {posA[0] - atoms[a].x, posA[1] - atoms[a].y, posA[2] - atoms[a].z};
    pbc(superBox, dr);
    double rr = std::max(0.1, dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    if (rr < rc2)
    {
      Factor v = gridFactor(grid_type, ff, rr, typeA, atoms[a]);
      energy += v.e;
      for (int i = 0; i != 3; ++i)
      {
        g[i] += dr[i] * v.f1;
        for (int j = 0; j != 3; ++j)
        {
          h[i][j] += v.f2 * dr[i] * dr[j] + (i == j ? v.f1 : 0.0);
          for (int k = 0; k != 3; ++k)
          {
            t[i][j][k] += v.f3 * dr[i] * dr[j] * dr[k] + (j == k ? v.f2 * dr[i] : 0.0) +
                          (i == k ? v.f2 * dr[j] : 0.0) + (i == j ? v.f2 * dr[k] : 0.0);
          }
        }
      }
    }
  }
}

void tricubicFractional(int grid_type, const off* ff, const Box& superBox, const double* posA, int typeA,
                        const Box& unitBox, const oatom* atoms, int n, double out[8])
{
  const double rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  if (!unitBox.triclinic)
  {
    // rectangular branch, framework_molecule_grid.cpp:192-243
    double energy = 0.0, fx = 0.0, fy = 0.0, fz = 0.0, fxy = 0.0, fxz = 0.0, fyz = 0.0, fxyz = 0.0;
    for (int a = 0; a < n; ++a)
    {
      double dr[3] = {posA[0] - atoms[a].x, posA[1] - atoms[a].y, posA[2] - atoms[a].z};
      pbc(superBox, dr);
      double rr = std::max(0.1, dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      if (rr < rc2)
      {
        Factor v = gridFactor(grid_type, ff, rr, typeA, atoms[a]);
        energy += v.e;
        fx += dr[0] * v.f1;
        fy += dr[1] * v.f1;
        fz += dr[2] * v.f1;
        fxy += v.f2 * dr[0] * dr[1];
        fxz += v.f2 * dr[0] * dr[2];
        fyz += v.f2 * dr[1] * dr[2];
        fxyz += v.f3 * dr[0] * dr[1] * dr[2];
      }
    }
    const double cx = unitBox.c[0][0], cy = unitBox.c[1][1], cz = unitBox.c[2][2];
    out[0] = energy;
    out[1] = fx * cx;
    out[2] = fy * cy;
    out[3] = fz * cz;
    out[4] = fxy * cx * cy;
    out[5] = fxz * cx * cz;
    out[6] = fyz * cy * cz;
    out[7] = fxyz * cx * cy * cz;
    return;
  }
  // triclinic branch, framework_molecule_grid.cpp:244-279
  double energy, g[3], h[3][3], t[3][3][3];
  tricubicCartesian(grid_type, ff, superBox, posA, typeA, atoms, n, energy, g, h, t);
  const auto& C = unitBox.c;  // C[row-vector index][p] = frameworkCell[index][p]
  double f[3] = {0, 0, 0}, s01 = 0, s02 = 0, s12 = 0, t012 = 0;
  for (int p = 0; p < 3; ++p)
  {
    f[0] += C[0][p] * g[p];
    f[1] += C[1][p] * g[p];
    f[2] += C[2][p] * g[p];
    for (int q = 0; q < 3; ++q)
    {
      s01 += C[0][p] * C[1][q] * h[p][q];
      s02 += C[0][p] * C[2][q] * h[p][q];
      s12 += C[1][p] * C[2][q] * h[p][q];
      for (int r = 0; r < 3; ++r) t012 += C[0][p] * C[1][q] * C[2][r] * t[p][q][r];
    }
  }
  out[0] = energy;
  out[1] = f[0];
  out[2] = f[1];
  out[3] = f[2];
  out[4] = s01;
  out[5] = s02;
  out[6] = s12;
  out[7] = t012;
}

struct GridSetup
{
  Box unit, super;
  std::vector<oatom> atoms;
  int ncx, ncy, ncz;
};

GridSetup gridSetup(const obox* unit_box, const oatom* unit_atoms, int n_unit, double cutoff, int nx, int ny, int nz)
{
  GridSetup s;
  s.unit = makeBox(unit_box);
  // SimulationBox::smallestNumberOfUnitCellsForMinimumImagesConvention (simulationbox.cpp:150-156)
  double w[3];
  perpendicularWidths(s.unit, w);
  int n[3];
  for (int d = 0; d < 3; ++d) n[d] = static_cast<int>(std::ceil(2.0 * cutoff / w[d]));
  // Framework::makeSuperCell(int3) (framework.cpp:1105-1127): i outer, k inner, atoms innermost
  for (int i = 0; i < n[0]; ++i)
    for (int j = 0; j < n[1]; ++j)
      for (int k = 0; k < n[2]; ++k)
        for (int a = 0; a < n_unit; ++a)
        {
          oatom c = unit_atoms[a];
          double f[3] = {static_cast<double>(i), static_cast<double>(j), static_cast<double>(k)}, d[3];
          matvec(s.unit.c, f, d);
          c.x += d[0];
          c.y += d[1];
          c.z += d[2];
          s.atoms.push_back(c);
        }
  s.super = scaledBox(s.unit, n[0], n[1], n[2]);
  s.ncx = nx - 1;
  s.ncy = ny - 1;
  s.ncz = nz - 1;
  return s;
}

// One grid point of makeFrameworkInterpolationGrid, tricubic branch (interpolation_energy_grid.cpp:3826-3874).
void gridPoint(int grid_type, const off* ff, const GridSetup& s, int probe_type, int64_t i, int64_t j, int64_t k,
               double* dst)
{
  double delta[3] = {1.0 / static_cast<double>(s.ncx), 1.0 / static_cast<double>(s.ncy),
                     1.0 / static_cast<double>(s.ncz)};
  double frac[3] = {static_cast<double>(i) * delta[0], static_cast<double>(j) * delta[1],
                    static_cast<double>(k) * delta[2]};
  double pos[3];
  matvec(s.unit.c, frac, pos);
  double values[8];
  tricubicFractional(grid_type, ff, s.super, pos, probe_type, s.unit, s.atoms.data(), static_cast<int>(s.atoms.size()),
                     values);
  const double cx = static_cast<double>(s.ncx), cy = static_cast<double>(s.ncy), cz = static_cast<double>(s.ncz);
  values[1] /= cx;
  values[2] /= cy;
  values[3] /= cz;
  values[4] /= cx * cy;
  values[5] /= cx * cz;
  values[6] /= cy * cz;
  values[7] /= cx * cy * cz;
  const double oc = ff->overlap_criteria;
  if (values[0] > oc)
  {
    dst[0] = 2.0 * oc;
    dst[1] = std::clamp(values[1], -oc, oc);
    dst[2] = std::clamp(values[2], -oc, oc);
    dst[3] = std::clamp(values[3], -oc, oc);
    for (int l = 4; l < 8; ++l) dst[l] = 0.0;
  }
  else
  {
    for (int l = 0; l < 8; ++l) dst[l] = values[l];
  }
}

// Tricubic coefficient matrix: inverse of the map from the 64 monomial coefficients a[i+4j+16k] to the 64 corner
// values X[8*v + corner] (v = f, fx, fy, fz, fxy, fxz, fyz, fxyz; corner bit 0 = x, bit 1 = y, bit 2 = z).
struct TricubicMatrix
{
  double m[64][64];
  TricubicMatrix()
  {
    static const int dv[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                 {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
    auto dmono = [](int p, int d, int x) -> double
    {
      // d-th derivative of t^p at t = x (x in {0,1})
      if (d > p) return 0.0;
      double c = 1.0;
      for (int q = 0; q < d; ++q) c *= static_cast<double>(p - q);
      if (x == 0) return (p == d) ? c : 0.0;
      return c;
    };
    double B[64][128];
    for (int v = 0; v < 8; ++v)
      for (int corner = 0; corner < 8; ++corner)
      {
        int row = 8 * v + corner;
        int x = corner & 1, y = (corner >> 1) & 1, z = (corner >> 2) & 1;
        for (int k = 0; k < 4; ++k)
          for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 4; ++i)
              B[row][i + 4 * j + 16 * k] = dmono(i, dv[v][0], x) * dmono(j, dv[v][1], y) * dmono(k, dv[v][2], z);
        for (int c = 0; c < 64; ++c) B[row][64 + c] = (c == row) ? 1.0 : 0.0;
      }
    // Gauss-Jordan with partial pivoting; the inverse has small integer entries and is rounded to them.
    for (int col = 0; col < 64; ++col)
    {
      int piv = col;
      for (int r = col + 1; r < 64; ++r)
        if (std::fabs(B[r][col]) > std::fabs(B[piv][col])) piv = r;
      if (piv != col)
        for (int c = 0; c < 128; ++c) std::swap(B[piv][c], B[col][c]);
      double p = B[col][col];
      for (int c = 0; c < 128; ++c) B[col][c] /= p;
      for (int r = 0; r < 64; ++r)
      {
        if (r == col) continue;
        double f = B[r][col];
        if (f == 0.0) continue;
        for (int c = 0; c < 128; ++c) B[r][c] -= f * B[col][c];
      }
    }
    for (int r = 0; r < 64; ++r)
      for (int c = 0; c < 64; ++c) m[r][c] = std::rint(B[r][64 + c]);
    // nonzero pattern per row: the reference evaluates the map unrolled over its ~1000 nonzeros
    // (interpolation_energy_grid.cpp:195-358), so the oracle does the same amount of work
    for (int r = 0; r < 64; ++r)
    {
      start[r] = static_cast<int>(nzc.size());
      for (int c = 0; c < 64; ++c)
        if (m[r][c] != 0.0)
        {
          nzc.push_back(c);
          nzv.push_back(m[r][c]);
        }
    }
    start[64] = static_cast<int>(nzc.size());
  }
  int start[65];
  std::vector<int> nzc;
  std::vector<double> nzv;
};

const TricubicMatrix& tricubicMatrix()
{
  static const TricubicMatrix tm;
  return tm;
}

// The 64 monomial coefficients of the cell holding pos and the local coordinates in it (InterpolationEnergyGrid::
// interpolate, tricubic branch, interpolation_energy_grid.cpp:3980-4118; the same steps as interpolateHessian,
// :4518-4571).
void tricubicCoefficients(const double* data, int nx, int ny, int nz, const Box& unit, const double* pos, double a[64],
                          double s[3])
{
  double sraw[3];
  matvec(unit.ic, pos, sraw);
  for (int d = 0; d < 3; ++d) s[d] = fract1(sraw[d]);
  const int ncx = nx - 1, ncy = ny - 1, ncz = nz - 1;
  int64_t x0 = std::min(static_cast<int64_t>(s[0] * static_cast<double>(ncx)), static_cast<int64_t>(ncx - 1));
  int64_t y0 = std::min(static_cast<int64_t>(s[1] * static_cast<double>(ncy)), static_cast<int64_t>(ncy - 1));
  int64_t z0 = std::min(static_cast<int64_t>(s[2] * static_cast<double>(ncz)), static_cast<int64_t>(ncz - 1));
  int64_t x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
  s[0] = (s[0] * static_cast<double>(ncx)) - static_cast<double>(x0);
  s[1] = (s[1] * static_cast<double>(ncy)) - static_cast<double>(y0);
  s[2] = (s[2] * static_cast<double>(ncz)) - static_cast<double>(z0);
  auto at = [&](int l, int64_t i, int64_t j, int64_t k) { return data[l + 8 * (i + nx * (j + ny * k))]; };
  double X[64];
  for (int l = 0; l != 8; ++l)
  {
    X[8 * l + 0] = at(l, x0, y0, z0);
    X[8 * l + 1] = at(l, x1, y0, z0);
    X[8 * l + 2] = at(l, x0, y1, z0);
    X[8 * l + 3] = at(l, x1, y1, z0);
    X[8 * l + 4] = at(l, x0, y0, z1);
    X[8 * l + 5] = at(l, x1, y0, z1);
    X[8 * l + 6] = at(l, x0, y1, z1);
    X[8 * l + 7] = at(l, x1, y1, z1);
  }
  const TricubicMatrix& T = tricubicMatrix();
  for (int r = 0; r < 64; ++r)
  {
    double acc = 0.0;
    for (int q = T.start[r]; q < T.start[r + 1]; ++q) acc += T.nzv[q] * X[T.nzc[q]];
    a[r] = acc;
  }
}

double interpolateTricubic(const double* data, int nx, int ny, int nz, const Box& unit, const double* pos)
{
  double a[64], s[3];
  tricubicCoefficients(data, nx, ny, nz, unit, pos, a, s);
  double value = 0.0;
  for (int k = 0; k != 4; ++k)
    for (int j = 0; j != 4; ++j)
      for (int i = 0; i != 4; ++i)
        value += a[i + 4 * j + 16 * k] * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k);
  return value;
}

// Value and Cartesian gradient (InterpolationEnergyGrid::interpolateHessian, tricubic branch,
// interpolation_energy_grid.cpp:4572-4590)
double interpolateTricubicGradient(const double* data, int nx, int ny, int nz, const Box& unit, const double* pos,
                                   double grad[3])
{
  double a[64], s[3];
  tricubicCoefficients(data, nx, ny, nz, unit, pos, a, s);
  const double nc[3] = {static_cast<double>(nx - 1), static_cast<double>(ny - 1), static_cast<double>(nz - 1)};
  double value = 0.0, g[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k != 4; ++k)
    for (int j = 0; j != 4; ++j)
      for (int i = 0; i != 4; ++i)
      {
        const double c = a[i + 4 * j + 16 * k];
        value += c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k);
        if (i > 0) g[0] += nc[0] * i * c * std::pow(s[0], i - 1) * std::pow(s[1], j) * std::pow(s[2], k);
        if (j > 0) g[1] += nc[1] * j * c * std::pow(s[0], i) * std::pow(s[1], j - 1) * std::pow(s[2], k);
        if (k > 0) g[2] += nc[2] * k * c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k - 1);
      }
  // inverseCell^T * g: with M = inverseCell stored column-major (ic[col][row]), (M^T g)_a = sum_b ic[a][b] g_b
  for (int a2 = 0; a2 < 3; ++a2) grad[a2] = unit.ic[a2][0] * g[0] + unit.ic[a2][1] * g[1] + unit.ic[a2][2] * g[2];
  return value;
}

// ---- triquintic scheme (27 values per grid point) ----
//
// Channel l of a triquintic grid point holds the mixed derivative of the energy of orders kQuinticOrder[l] along the
// three lattice directions; the order list follows the divisors of makeFrameworkInterpolationGrid's triquintic branch
// (interpolation_energy_grid.cpp:3882-3945).
constexpr int kQuinticOrder[27][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {1, 0, 1},
                                      {0, 2, 0}, {0, 1, 1}, {0, 0, 2}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {1, 1, 1},
                                      {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {2, 1, 1},
                                      {1, 2, 1}, {1, 1, 2}, {2, 2, 1}, {2, 1, 2}, {1, 2, 2}, {2, 2, 2}};

// F[k] = (1/r d/dr)^k U(r), k = 0..6
struct Factor6
{
  double f[7];
};

// potentialLennardJonesTriquinticDerivative (potentials/interpolation/triquintic_derivative_lj.ixx:33-51). The
// reference's triquintic branch uses it for the repulsion and attraction grid types too
// (interactions/framework_molecule_grid.cpp:584-592).
inline Factor6 ljTriquintic(double eps, double sigma, double shift, double r2)
{
  const double arg1 = 4.0 * eps;
  const double arg2 = sigma * sigma;
  const double temp3 = (arg2 / r2) * (arg2 / r2) * (arg2 / r2);
  const double r4 = r2 * r2, r6 = r4 * r2, r8 = r6 * r2, r10 = r8 * r2, r12 = r10 * r2;
  const double t6 = temp3 * temp3;
  return {{arg1 * (t6 - temp3) - shift, -6.0 * arg1 * (2.0 * t6 - temp3) / r2, 24.0 * arg1 * (7.0 * t6 - 2.0 * temp3) / r4,
           -96.0 * arg1 * (28.0 * t6 - 5.0 * temp3) / r6, 1152.0 * arg1 * (42.0 * t6 - 5.0 * temp3) / r8,
           -80640.0 * arg1 * (12.0 * t6 - temp3) / r10, 645120.0 * arg1 * (33.0 * t6 - 2.0 * temp3) / r12}};
}

// potentialRealEwaldTriquinticDerivative (potentials/interpolation/triquintic_derivative_real_ewald.ixx:32-78)
inline Factor6 ewaldTriquintic(double alpha, double rr, double r, double qa, double qb)
{
  const double Cq = coulombFactor() * qa * qb;
  const double ec = std::erfc(alpha * r);
  const double et = 2.0 * alpha * r * std::exp(-alpha * alpha * rr) * kInvSqrtPi;
  const double a2 = (alpha * r) * (alpha * r), a4 = a2 * a2, a6 = a4 * a2, a8 = a6 * a2, a10 = a8 * a2;
  const double r3 = rr * r, r5 = r3 * rr, r7 = r5 * rr, r9 = r7 * rr, r11 = r9 * rr, r13 = r11 * rr;
  return {{Cq * ec / r, -Cq * ((et + ec) / r3), Cq * ((et * (2.0 * a2 + 3.0) + 3.0 * ec) / r5),
           -Cq * ((et * (4.0 * a4 + 10.0 * a2 + 15.0) + 15.0 * ec) / r7),
           Cq * ((et * (8.0 * a6 + 28.0 * a4 + 70.0 * a2 + 105.0) + 105.0 * ec) / r9),
           -Cq * ((et * (16.0 * a8 + 72.0 * a6 + 252.0 * a4 + 630.0 * a2 + 945.0) + 945.0 * ec) / r11),
           Cq * ((et * (32.0 * a10 + 176.0 * a8 + 792.0 * a6 + 2772.0 * a4 + 6930.0 * a2 + 10395.0) + 10395.0 * ec) /
                 r13)}};
}

inline Factor6 quinticFactor(int grid_type, const off* ff, double rr, int typeA, const oatom& b)
{
  if (grid_type == 1) return ewaldTriquintic(ff->ewald_alpha, rr, std::sqrt(rr), 1.0, b.charge);
  const int idx = typeA * ff->n_types + b.type;
  return ljTriquintic(ff->epsilon[idx], ff->sigma[idx], ff->shift[idx], rr);
}

// d^n/dx^n of a radial function along one Cartesian axis, as a polynomial in x and the factors F:
// sum over m pairs of n!/(m! 2^m (n-2m)!) x^(n-2m) F[n-m]. The mixed Cartesian derivative of orders (i, j, k) is the
// product of the three axis polynomials with the F indices added up (every derivative of a radial function is a sum
// over partial pairings of its directions: each pair gives a Kronecker delta, each unpaired direction a component of
// dr, and F takes the index directions - pairs).
double cartesianDerivative(int i, int j, int k, const double dr[3], const double F[7])
{
  auto terms = [](int n, double x, double* c, int* fk, int& cnt)
  {
    cnt = 0;
    for (int m = 0; 2 * m <= n; ++m)
    {
      double coef = 1.0;
      for (int q = 0; q < n; ++q) coef *= static_cast<double>(q + 1);  // n!
      double den = 1.0;
      for (int q = 0; q < m; ++q) den *= static_cast<double>(q + 1) * 2.0;  // m! 2^m
      for (int q = 0; q < n - 2 * m; ++q) den *= static_cast<double>(q + 1);  // (n-2m)!
      c[cnt] = coef / den * std::pow(x, n - 2 * m);
      fk[cnt] = n - m;
      ++cnt;
    }
  };
  double cx[4], cy[4], cz[4];
  int kx[4], ky[4], kz[4], nx, ny, nz;
  terms(i, dr[0], cx, kx, nx);
  terms(j, dr[1], cy, ky, ny);
  terms(k, dr[2], cz, kz, nz);
  double v = 0.0;
  for (int a = 0; a < nx; ++a)
    for (int b = 0; b < ny; ++b)
      for (int c = 0; c < nz; ++c) v += cx[a] * cy[b] * cz[c] * F[kx[a] + ky[b] + kz[c]];
  return v;
}

// Interactions::calculateTriquinticFractionalAtPosition (interactions/framework_molecule_grid.cpp:549-813).
// Rectangular cells (:568-683): the 27 Cartesian mixed derivatives summed over the supercell atoms, scaled by the cell
// diagonal. With reference_rectangular the two deviations of that branch are kept: the first derivatives along y and
// z are scaled by cell[0][0] (:648-650), and the (2,2,2) channel lacks its F3 term (:671-676). Without it the branch
// gives the exact derivatives, the values of the triclinic branch for the same cell.
// Triclinic cells (:684-812, with calculateTriquinticDerivativeAtPosition :284-503): the full Cartesian derivative
// tensors summed over the atoms, then contracted with the cell vectors.
void triquinticFractional(int grid_type, const off* ff, const Box& superBox, const double* posA, int typeA,
                          const Box& unitBox, const oatom* atoms, int n, bool reference_rectangular, double out[27])
{
  const double rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  // Cartesian derivative sums by multiset (i x's, j y's, k z's), i + j + k <= 6
  double T[7][7][7];
  std::memset(T, 0, sizeof(T));
  double sumF3 = 0.0;
  for (int a = 0; a < n; ++a)
  {
    double dr[3] = {posA[0] - atoms[a].x, posA[1] - atoms[a].y, posA[2] - atoms[a].z};
    pbc(superBox, dr);
    const double rr = std::max(0.1, dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    if (rr >= rc2) continue;
    const Factor6 v = quinticFactor(grid_type, ff, rr, typeA, atoms[a]);
    sumF3 += v.f[3];
    for (int i = 0; i <= 6; ++i)
      for (int j = 0; i + j <= 6; ++j)
        for (int k = 0; i + j + k <= 6; ++k) T[i][j][k] += cartesianDerivative(i, j, k, dr, v.f);
  }
  const auto& C = unitBox.c;  // C[a][p]: component p of lattice vector a
  if (!unitBox.triclinic)
  {
    for (int l = 0; l < 27; ++l)
    {
      const int* o = kQuinticOrder[l];
      out[l] = T[o[0]][o[1]][o[2]] * std::pow(C[0][0], o[0]) * std::pow(C[1][1], o[1]) * std::pow(C[2][2], o[2]);
    }
    if (reference_rectangular)
    {
      out[2] = T[0][1][0] * C[0][0];
      out[3] = T[0][0][1] * C[0][0];
      out[26] -= sumF3 * C[0][0] * C[0][0] * C[1][1] * C[1][1] * C[2][2] * C[2][2];
    }
    return;
  }
  // contraction: sum over Cartesian index tuples p_1..p_n of prod_t C[d_t][p_t] * T[multiset(p)]
  for (int l = 0; l < 27; ++l)
  {
    const int* o = kQuinticOrder[l];
    int dirs[6], nd = 0;
    for (int ax = 0; ax < 3; ++ax)
      for (int q = 0; q < o[ax]; ++q) dirs[nd++] = ax;
    int total = 1;
    for (int q = 0; q < nd; ++q) total *= 3;
    double acc = 0.0;
    for (int code = 0; code < total; ++code)
    {
      int cnt[3] = {0, 0, 0}, c = code;
      double w = 1.0;
      for (int q = 0; q < nd; ++q)
      {
        const int p = c % 3;
        c /= 3;
        ++cnt[p];
        w *= C[dirs[q]][p];
      }
      acc += w * T[cnt[0]][cnt[1]][cnt[2]];
    }
    out[l] = acc;
  }
}

// One grid point of makeFrameworkInterpolationGrid, triquintic branch (interpolation_energy_grid.cpp:3882-3962).
void gridPointQuintic(int grid_type, const off* ff, const GridSetup& s, int probe_type, int64_t i, int64_t j, int64_t k,
                      bool reference_rectangular, double* dst)
{
  const double delta[3] = {1.0 / static_cast<double>(s.ncx), 1.0 / static_cast<double>(s.ncy),
                           1.0 / static_cast<double>(s.ncz)};
  const double frac[3] = {static_cast<double>(i) * delta[0], static_cast<double>(j) * delta[1],
                          static_cast<double>(k) * delta[2]};
  double pos[3];
  matvec(s.unit.c, frac, pos);
  double values[27];
  triquinticFractional(grid_type, ff, s.super, pos, probe_type, s.unit, s.atoms.data(),
                       static_cast<int>(s.atoms.size()), reference_rectangular, values);
  const double nc[3] = {static_cast<double>(s.ncx), static_cast<double>(s.ncy), static_cast<double>(s.ncz)};
  for (int l = 1; l < 27; ++l)
  {
    const int* o = kQuinticOrder[l];
    values[l] /= std::pow(nc[0], o[0]) * std::pow(nc[1], o[1]) * std::pow(nc[2], o[2]);
  }
  const double oc = ff->overlap_criteria;
  if (values[0] > oc)
  {
    dst[0] = 2.0 * oc;
    dst[1] = std::clamp(values[1], -oc, oc);
    dst[2] = std::clamp(values[2], -oc, oc);
    dst[3] = std::clamp(values[3], -oc, oc);
    for (int l = 4; l < 27; ++l) dst[l] = 0.0;
  }
  else
  {
    for (int l = 0; l < 27; ++l) dst[l] = values[l];
  }
}

// Triquintic coefficient map: inverse of the map from the 216 monomial coefficients a[i + 6j + 36k] to the corner data
// X[8*l + corner] (channel l of kQuinticOrder, corner bit 0 = x, bit 1 = y, bit 2 = z), regenerated by Gauss-Jordan
// elimination. 8 times each entry is an integer (the reference stores those integers and scales by 0.125,
// interpolation_energy_grid.cpp:360, 4160-4164); the oracle rounds to them.
struct TriquinticMatrix
{
  std::vector<double> m;  // 216 x 216
  std::vector<int> start, nzc;
  std::vector<double> nzv;
  TriquinticMatrix() : m(216 * 216), start(217)
  {
    auto dmono = [](int p, int d, int x) -> double
    {
      if (d > p) return 0.0;
      double c = 1.0;
      for (int q = 0; q < d; ++q) c *= static_cast<double>(p - q);
      if (x == 0) return (p == d) ? c : 0.0;
      return c;
    };
    const int N = 216;
    std::vector<double> B(static_cast<size_t>(N) * 2 * N, 0.0);
    auto b = [&](int r, int c) -> double& { return B[static_cast<size_t>(r) * 2 * N + c]; };
    for (int l = 0; l < 27; ++l)
      for (int corner = 0; corner < 8; ++corner)
      {
        const int row = 8 * l + corner;
        const int x = corner & 1, y = (corner >> 1) & 1, z = (corner >> 2) & 1;
        for (int k = 0; k < 6; ++k)
          for (int j = 0; j < 6; ++j)
            for (int i = 0; i < 6; ++i)
              b(row, i + 6 * j + 36 * k) = dmono(i, kQuinticOrder[l][0], x) * dmono(j, kQuinticOrder[l][1], y) *
                                           dmono(k, kQuinticOrder[l][2], z);
        b(row, N + row) = 1.0;
      }
    for (int col = 0; col < N; ++col)
    {
      int piv = col;
      for (int r = col + 1; r < N; ++r)
        if (std::fabs(b(r, col)) > std::fabs(b(piv, col))) piv = r;
      if (piv != col)
        for (int c = 0; c < 2 * N; ++c) std::swap(b(piv, c), b(col, c));
      const double p = b(col, col);
      for (int c = 0; c < 2 * N; ++c) b(col, c) /= p;
      for (int r = 0; r < N; ++r)
      {
        if (r == col) continue;
        const double f = b(r, col);
        if (f == 0.0) continue;
        for (int c = 0; c < 2 * N; ++c) b(r, c) -= f * b(col, c);
      }
    }
    for (int r = 0; r < N; ++r)
    {
      start[r] = static_cast<int>(nzc.size());
      for (int c = 0; c < N; ++c)
      {
        const double v = 0.125 * std::rint(8.0 * b(r, N + c));
        m[static_cast<size_t>(r) * N + c] = v;
        if (v != 0.0)
        {
          nzc.push_back(c);
          nzv.push_back(v);
        }
      }
    }
    start[N] = static_cast<int>(nzc.size());
  }
};

const TriquinticMatrix& triquinticMatrix()
{
  static const TriquinticMatrix tm;
  return tm;
}

// Value and d/ds of sum_ijk a[i + 6j + 36k] s_x^i s_y^j s_z^k (the triquintic branch of interpolate and
// interpolateGradient, interpolation_energy_grid.cpp:4119-4178, 4348-4410) from the corner data X.
double quinticFromCorners(const double X[216], const double s[3], double ds[3])
{
  const TriquinticMatrix& T = triquinticMatrix();
  double a[216];
  for (int r = 0; r < 216; ++r)
  {
    double acc = 0.0;
    for (int q = T.start[r]; q < T.start[r + 1]; ++q) acc += T.nzv[q] * X[T.nzc[q]];
    a[r] = acc;
  }
  double value = 0.0;
  ds[0] = ds[1] = ds[2] = 0.0;
  for (int i = 0; i != 6; ++i)
    for (int j = 0; j != 6; ++j)
      for (int k = 0; k != 6; ++k)
      {
        const double c = a[i + 6 * j + 36 * k];
        value += c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k);
        if (i > 0) ds[0] += i * c * std::pow(s[0], i - 1) * std::pow(s[1], j) * std::pow(s[2], k);
        if (j > 0) ds[1] += j * c * std::pow(s[0], i) * std::pow(s[1], j - 1) * std::pow(s[2], k);
        if (k > 0) ds[2] += k * c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k - 1);
      }
  return value;
}

// Value, d/ds and d2/(ds_a ds_b) (h[0..5]: xx, xy, xz, yy, yz, zz) of the triquintic cell polynomial from the corner
// data X (the triquintic branch of interpolateHessian, interpolation_energy_grid.cpp:4602-4745)
double quinticFromCornersHessian(const double X[216], const double s[3], double ds[3], double h[6])
{
  const TriquinticMatrix& T = triquinticMatrix();
  double a[216];
  for (int r = 0; r < 216; ++r)
  {
    double acc = 0.0;
    for (int q = T.start[r]; q < T.start[r + 1]; ++q) acc += T.nzv[q] * X[T.nzc[q]];
    a[r] = acc;
  }
  // powers and their first and second derivatives per axis
  double pw[3][6], d1[3][6], d2[3][6];
  for (int ax = 0; ax < 3; ++ax)
    for (int e = 0; e < 6; ++e)
    {
      pw[ax][e] = std::pow(s[ax], e);
      d1[ax][e] = e > 0 ? e * std::pow(s[ax], e - 1) : 0.0;
      d2[ax][e] = e > 1 ? e * (e - 1) * std::pow(s[ax], e - 2) : 0.0;
    }
  double value = 0.0;
  for (int q = 0; q < 3; ++q) ds[q] = 0.0;
  for (int q = 0; q < 6; ++q) h[q] = 0.0;
  for (int i = 0; i != 6; ++i)
    for (int j = 0; j != 6; ++j)
      for (int k = 0; k != 6; ++k)
      {
        const double c = a[i + 6 * j + 36 * k];
        value += c * pw[0][i] * pw[1][j] * pw[2][k];
        ds[0] += c * d1[0][i] * pw[1][j] * pw[2][k];
        ds[1] += c * pw[0][i] * d1[1][j] * pw[2][k];
        ds[2] += c * pw[0][i] * pw[1][j] * d1[2][k];
        h[0] += c * d2[0][i] * pw[1][j] * pw[2][k];
        h[1] += c * d1[0][i] * d1[1][j] * pw[2][k];
        h[2] += c * d1[0][i] * pw[1][j] * d1[2][k];
        h[3] += c * pw[0][i] * d2[1][j] * pw[2][k];
        h[4] += c * pw[0][i] * d1[1][j] * d1[2][k];
        h[5] += c * pw[0][i] * pw[1][j] * d2[2][k];
      }
  return value;
}

// Cartesian gradient and Hessian from derivatives along the cell axes: grad = M^T g, H = M^T Hs M with M the inverse
// cell (interpolation_energy_grid.cpp:4745-4748, system_interpolation_grids.cpp:336-350)
void toCartesian(const Box& unit, const double g[3], const double hs[6], double grad[3], double hc[6])
{
  const double Hs[3][3] = {{hs[0], hs[1], hs[2]}, {hs[1], hs[3], hs[4]}, {hs[2], hs[4], hs[5]}};
  for (int i = 0; i < 3; ++i) grad[i] = unit.ic[i][0] * g[0] + unit.ic[i][1] * g[1] + unit.ic[i][2] * g[2];
  const int pairs[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  for (int q = 0; q < 6; ++q)
  {
    const int i = pairs[q][0], j = pairs[q][1];
    double acc = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) acc += unit.ic[i][a] * unit.ic[j][b] * Hs[a][b];
    hc[q] = acc;
  }
}

// interpolateHessian, triquintic branch: value, Cartesian gradient and Hessian
double interpolateTriquinticHessian(const double* data, int nx, int ny, int nz, const Box& unit, const double* pos,
                                    double grad[3], double hess[6])
{
  double sraw[3], s[3];
  matvec(unit.ic, pos, sraw);
  for (int d = 0; d < 3; ++d) s[d] = fract1(sraw[d]);
  const int nc[3] = {nx - 1, ny - 1, nz - 1};
  int64_t i0[3];
  for (int d = 0; d < 3; ++d)
  {
    i0[d] = std::min(static_cast<int64_t>(s[d] * static_cast<double>(nc[d])), static_cast<int64_t>(nc[d] - 1));
    s[d] = s[d] * static_cast<double>(nc[d]) - static_cast<double>(i0[d]);
  }
  double X[216];
  for (int l = 0; l < 27; ++l)
    for (int corner = 0; corner < 8; ++corner)
    {
      const int64_t x = i0[0] + (corner & 1), y = i0[1] + ((corner >> 1) & 1), z = i0[2] + ((corner >> 2) & 1);
      X[8 * l + corner] = data[l + 27 * (x + nx * (y + ny * z))];
    }
  double ds[3], hs[6];
  const double value = quinticFromCornersHessian(X, s, ds, hs);
  const double g[3] = {ds[0] * nc[0], ds[1] * nc[1], ds[2] * nc[2]};
  const int pairs[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  double h[6];
  for (int q = 0; q < 6; ++q) h[q] = hs[q] * nc[pairs[q][0]] * nc[pairs[q][1]];
  toCartesian(unit, g, h, grad, hess);
  return value;
}

// The same for the tricubic map (a[i + 4j + 16k], X[8*v + corner])
double cubicFromCorners(const double X[64], const double s[3], double ds[3])
{
  const TricubicMatrix& T = tricubicMatrix();
  double a[64];
  for (int r = 0; r < 64; ++r)
  {
    double acc = 0.0;
    for (int q = T.start[r]; q < T.start[r + 1]; ++q) acc += T.nzv[q] * X[T.nzc[q]];
    a[r] = acc;
  }
  double value = 0.0;
  ds[0] = ds[1] = ds[2] = 0.0;
  for (int k = 0; k != 4; ++k)
    for (int j = 0; j != 4; ++j)
      for (int i = 0; i != 4; ++i)
      {
        const double c = a[i + 4 * j + 16 * k];
        value += c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k);
        if (i > 0) ds[0] += i * c * std::pow(s[0], i - 1) * std::pow(s[1], j) * std::pow(s[2], k);
        if (j > 0) ds[1] += j * c * std::pow(s[0], i) * std::pow(s[1], j - 1) * std::pow(s[2], k);
        if (k > 0) ds[2] += k * c * std::pow(s[0], i) * std::pow(s[1], j) * std::pow(s[2], k - 1);
      }
  return value;
}

// InterpolationEnergyGrid::interpolate / interpolateGradient, triquintic branch: the cell of pos, its 216 corner
// values, the polynomial; the gradient mapped to Cartesian with the inverse cell (interpolation_energy_grid.cpp:4410).
double interpolateTriquintic(const double* data, int nx, int ny, int nz, const Box& unit, const double* pos,
                             double grad[3])
{
  double sraw[3], s[3];
  matvec(unit.ic, pos, sraw);
  for (int d = 0; d < 3; ++d) s[d] = fract1(sraw[d]);
  const int nc[3] = {nx - 1, ny - 1, nz - 1};
  int64_t i0[3];
  for (int d = 0; d < 3; ++d)
  {
    i0[d] = std::min(static_cast<int64_t>(s[d] * static_cast<double>(nc[d])), static_cast<int64_t>(nc[d] - 1));
    s[d] = s[d] * static_cast<double>(nc[d]) - static_cast<double>(i0[d]);
  }
  double X[216];
  for (int l = 0; l < 27; ++l)
    for (int corner = 0; corner < 8; ++corner)
    {
      const int64_t x = i0[0] + (corner & 1), y = i0[1] + ((corner >> 1) & 1), z = i0[2] + ((corner >> 2) & 1);
      X[8 * l + corner] = data[l + 27 * (x + nx * (y + ny * z))];
    }
  double ds[3];
  const double value = quinticFromCorners(X, s, ds);
  if (grad)
  {
    const double g[3] = {ds[0] * nc[0], ds[1] * nc[1], ds[2] * nc[2]};
    for (int a = 0; a < 3; ++a) grad[a] = unit.ic[a][0] * g[0] + unit.ic[a][1] * g[1] + unit.ic[a][2] * g[2];
  }
  return value;
}

inline int groupOf(const oatom& a) { return a.group_fractional & 0x0f; }
inline bool fractionalOf(const oatom& a) { return (a.group_fractional >> 4) != 0; }

inline void addDud(double* arr, int gA, int gB, double sA, double sB, double factor)
{
  // RunningEnergy::addDudlambda* (running_energy.ixx:258-279)
  if (gA != 0) arr[gA - 1] += sB * factor;
  if (gB != 0) arr[gB - 1] += sA * factor;
}

void pairVDW(const off* ff, double sA, double sB, double rr, int tA, int tB, double out[2])
{
  // potentialVDW<0>, Lennard-Jones branch (potentials/pair_vdw.ixx:85-101); other types -> zero
  int idx = tA * ff->n_types + tB;
  if (!ff->lj[idx])
  {
    out[0] = 0.0;
    out[1] = 0.0;
    return;
  }
  double scaling = sA * sB;
  double arg1 = 4.0 * ff->epsilon[idx];
  double arg2 = ff->sigma[idx] * ff->sigma[idx];
  double arg3 = ff->shift[idx];
  double temp = (rr / arg2);
  double temp3 = temp * temp * temp;
  double inv_scaling = 1.0 - scaling;
  double rri3 = 1.0 / (temp3 + 0.5 * inv_scaling * inv_scaling);
  double rri6 = rri3 * rri3;
  double term = arg1 * (rri3 * (rri3 - 1.0)) - arg3;
  double dlambda_term = arg1 * scaling * inv_scaling * (2.0 * rri6 * rri3 - rri6);
  out[0] = scaling * term;
  out[1] = term + dlambda_term;
}

void pairCoulomb(const off* ff, double sA, double sB, double r, double qA, double qB, double out[2])
{
  // potentialCoulomb<0>, Ewald branch (potentials/pair_coulomb.ixx:51-77)
  double scaling = sA * sB;
  double alpha = ff->ewald_alpha;
  double prefactor = coulombFactor() * qA * qB;
  double s = r + 0.01 * (1.0 - scaling);
  double inverseS = 1.0 / s;
  double inverseSS = inverseS * inverseS;
  double erfcTerm = std::erfc(alpha * s);
  double gaussian = std::exp(-alpha * alpha * s * s) * kInvSqrtPi;
  double phi = erfcTerm * inverseS;
  double phiPrime = -(erfcTerm * inverseSS + 2.0 * alpha * gaussian * inverseS);
  out[0] = scaling * prefactor * phi;
  out[1] = prefactor * (phi - scaling * 0.01 * phiPrime);
}

// ---- Ewald (interactions/ewald.cpp, interactions/ewald_kvector.ixx) ----
struct Cplx
{
  double re, im;
};
inline Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cplx conjIf(Cplx a, bool c) { return c ? Cplx{a.re, -a.im} : a; }
inline double norm2(Cplx a) { return a.re * a.re + a.im * a.im; }

struct EikTables
{
  int n, kx, ky, kz;
  std::vector<Cplx> x, y, z;
  // Ewald::buildEikTables (ewald_kvector.ixx): atom-major eik_x[i + kx*N], k = 0,1 explicit, then recurrence
  EikTables(const Box& b, const std::vector<const oatom*>& atoms, int kxm, int kym, int kzm)
      : n(static_cast<int>(atoms.size())), kx(kxm), ky(kym), kz(kzm)
  {
    x.resize(static_cast<size_t>(n) * (kxm + 1));
    y.resize(static_cast<size_t>(n) * (kym + 1));
    z.resize(static_cast<size_t>(n) * (kzm + 1));
    for (int i = 0; i < n; ++i)
    {
      x[i] = y[i] = z[i] = Cplx{1.0, 0.0};
      double p[3] = {atoms[i]->x, atoms[i]->y, atoms[i]->z}, s[3];
      matvec(b.ic, p, s);
      for (int d = 0; d < 3; ++d) s[d] *= 2.0 * kPi;
      if (kxm >= 1) x[i + n] = Cplx{std::cos(s[0]), std::sin(s[0])};
      if (kym >= 1) y[i + n] = Cplx{std::cos(s[1]), std::sin(s[1])};
      if (kzm >= 1) z[i + n] = Cplx{std::cos(s[2]), std::sin(s[2])};
    }
    for (int k = 2; k <= kxm; ++k)
      for (int i = 0; i < n; ++i) x[i + k * n] = cmul(x[i + (k - 1) * n], x[i + n]);
    for (int k = 2; k <= kym; ++k)
      for (int i = 0; i < n; ++i) y[i + k * n] = cmul(y[i + (k - 1) * n], y[i + n]);
    for (int k = 2; k <= kzm; ++k)
      for (int i = 0; i < n; ++i) z[i + k * n] = cmul(z[i + (k - 1) * n], z[i + n]);
  }
  // fillEikXYRow + eikPhase
  Cplx xy(int i, int kxv, int kyv) const { return cmul(x[i + n * kxv], conjIf(y[i + n * std::abs(kyv)], kyv < 0)); }
  Cplx zf(int i, int kzv) const { return conjIf(z[i + n * std::abs(kzv)], kzv < 0); }
};

// Iterates the k-vectors in the reference order, calling body(kx, ky, kz, rksq, factor) for each accepted one.
template <typename F>
void forEachK(const off* ff, const Box& b, F&& body)
{
  double ax[3] = {b.ic[0][0], b.ic[1][0], b.ic[2][0]};
  double ay[3] = {b.ic[0][1], b.ic[1][1], b.ic[2][1]};
  double az[3] = {b.ic[0][2], b.ic[1][2], b.ic[2][2]};
  const double prefactor = coulombFactor() * (2.0 * kPi / b.volume);
  for (int kx = 0; kx <= ff->kmax_x; ++kx)
  {
    double kvx[3];
    for (int d = 0; d < 3; ++d) kvx[d] = 2.0 * kPi * static_cast<double>(kx) * ax[d];
    double factor = (kx == 0) ? (1.0 * prefactor) : (2.0 * prefactor);
    for (int ky = -ff->kmax_y; ky <= ff->kmax_y; ++ky)
    {
      double kvy[3];
      for (int d = 0; d < 3; ++d) kvy[d] = 2.0 * kPi * static_cast<double>(ky) * ay[d];
      for (int kz = -ff->kmax_z; kz <= ff->kmax_z; ++kz)
      {
        double kvz[3];
        for (int d = 0; d < 3; ++d) kvz[d] = 2.0 * kPi * static_cast<double>(kz) * az[d];
        double kv[3] = {kvx[0] + kvy[0] + kvz[0], kvx[1] + kvy[1] + kvz[1], kvx[2] + kvy[2] + kvz[2]};
        double rksq = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        uint64_t ksq = static_cast<uint64_t>(kx * kx + ky * ky + kz * kz);
        if ((ksq != 0) && (ksq <= ff->recip_int_cutoff_sq) && (rksq < ff->recip_cutoff_sq))
          body(kx, ky, kz, rksq, factor);
      }
    }
  }
}

// Potentials::ewaldExclusionFactors (potentials/coulomb_real_space.ixx:49-65): potential and dU/dlambda factor
inline void exclusionFactors(double alpha, double scalingTotal, double r, double& potential, double& dudl)
{
  const double offset = 0.01 * (1.0 - scalingTotal);
  const double s = r + offset;
  const double inverseS = 1.0 / s;
  potential = std::erf(alpha * s) * inverseS;
  const double gaussianTerm = 2.0 * alpha * kInvSqrtPi * std::exp(-alpha * alpha * s * s);
  const double firstDerivative = (gaussianTerm - potential) * inverseS;
  dudl = potential - scalingTotal * 0.01 * firstDerivative;
}

void addFourierDUdlambda(oenergy* e, double factor, Cplx sk, const Cplx* dsk)
{
  // ewald.cpp:166-173
  for (int g = 0; g != 4; ++g) e->dudlambda_ewald[g] += factor * (sk.re * dsk[g].re + sk.im * dsk[g].im);
}

}  // namespace

extern "C"
{
double oracle_energy_to_kelvin(void) { return energyConversionFactor() * kAvogadroConstant / kMolarGasConstant; }
double oracle_kelvin_to_energy(void) { return kMolarGasConstant / (energyConversionFactor() * kAvogadroConstant); }
double oracle_coulomb_factor(void) { return coulombFactor(); }

void oracle_tricubic_fractional_at_position(int grid_type, const off* ff, const obox* super_box, const double* pos,
                                            int type_a, const obox* unit_box, const oatom* super_atoms, int n,
                                            double out[8])
{
  Box sb = makeBox(super_box), ub = makeBox(unit_box);
  tricubicFractional(grid_type, ff, sb, pos, type_a, ub, super_atoms, n, out);
}

int oracle_make_tricubic_grid(int grid_type, const off* ff, const obox* unit_box, const oatom* unit_atoms, int n_unit,
                              int probe_type, double cutoff, int nx, int ny, int nz, const int64_t* points,
                              int64_t n_points, int threads, double* out)
{
  GridSetup s = gridSetup(unit_box, unit_atoms, n_unit, cutoff, nx, ny, nz);
  const int64_t total = points ? n_points : static_cast<int64_t>(nx) * ny * nz;
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
#endif
  for (int64_t p = 0; p < total; ++p)
  {
    int64_t flat = points ? points[p] : p;
    int64_t i = flat % nx, j = (flat / nx) % ny, k = flat / (static_cast<int64_t>(nx) * ny);
    double* dst = points ? out + 8 * p : out + 8 * flat;
    gridPoint(grid_type, ff, s, probe_type, i, j, k, dst);
  }
  (void)threads;
  return static_cast<int>(s.atoms.size());
}

int64_t oracle_grid_pair_count(int grid_type, const off* ff, const obox* unit_box, const oatom* unit_atoms, int n_unit,
                               int probe_type, double cutoff, int nx, int ny, int nz, const int64_t* points,
                               int64_t n_points, int threads)
{
  GridSetup s = gridSetup(unit_box, unit_atoms, n_unit, cutoff, nx, ny, nz);
  const int64_t total = points ? n_points : static_cast<int64_t>(nx) * ny * nz;
  const double rc2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  std::vector<char> active(s.atoms.size());
  for (size_t a = 0; a < s.atoms.size(); ++a)
  {
    const oatom& b = s.atoms[a];
    active[a] = (grid_type == 1) ? (b.charge != 0.0) : (ff->epsilon[probe_type * ff->n_types + b.type] != 0.0);
  }
  int64_t count = 0;
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : count) num_threads(threads)
#endif
  for (int64_t p = 0; p < total; ++p)
  {
    int64_t flat = points ? points[p] : p;
    int64_t i = flat % nx, j = (flat / nx) % ny, k = flat / (static_cast<int64_t>(nx) * ny);
    double frac[3] = {static_cast<double>(i) / s.ncx, static_cast<double>(j) / s.ncy, static_cast<double>(k) / s.ncz};
    double pos[3];
    matvec(s.unit.c, frac, pos);
    for (size_t a = 0; a < s.atoms.size(); ++a)
    {
      if (!active[a]) continue;
      double dr[3] = {pos[0] - s.atoms[a].x, pos[1] - s.atoms[a].y, pos[2] - s.atoms[a].z};
      pbc(s.super, dr);
      double rr = std::max(0.1, dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      if (rr < rc2) ++count;
    }
  }
  (void)threads;
  return count;
}

void oracle_tricubic_matrix(double* m)
{
  const auto& M = tricubicMatrix().m;
  for (int r = 0; r < 64; ++r)
    for (int c = 0; c < 64; ++c) m[64 * r + c] = M[r][c];
}

double oracle_grid_interpolate(const double* data, int nx, int ny, int nz, const obox* unit_box, const double* pos)
{
  Box ub = makeBox(unit_box);
  return interpolateTricubic(data, nx, ny, nz, ub, pos);
}

void oracle_grid_validate(const off* ff, const obox* unit_box, const oatom* unit_atoms, int n_unit,
                          const obox* simulation_box, int probe_type, int nx, int ny, int nz, const double* vdw_grid,
                          const double* ewald_grid, double probe_charge, double weight_beta, const double* points,
                          int64_t n_points, double* out)
{
  // System::createFrameworkInterpolationGrids, grid test of the tricubic scheme (system_interpolation_grids.cpp:272-651):
  // at each point (fractions of the simulation box) the interpolated and the analytical energy and Cartesian gradient
  // in K, Boltzmann weight exp(-weight_beta * E_vdw[K]); the charge term (probe charge x unit-charge Ewald grid) only
  // where the analytical VDW energy is below the overlap criterion. out: the 34 weighted sums and the two counts.
  const GridSetup gs = gridSetup(unit_box, unit_atoms, n_unit, ff->cutoff_framework_vdw, nx, ny, nz);
  const Box sim = makeBox(simulation_box);
  const double toK = energyConversionFactor() * kAvogadroConstant / kMolarGasConstant;
  for (int i = 0; i < 36; ++i) out[i] = 0.0;
  auto accumulate = [&](double* o, double w, double ei, double ef, const double* gi, const double* gf)
  {
    o[0] += w;
    o[1] += ei * w;
    o[2] += ef * w;
    o[3] += (ef - ei) * (ef - ei) * w;
    o[4] += ef * ef * w;
    for (int a = 0; a < 3; ++a)
    {
      o[5 + a] += gi[a] * w;
      o[8 + a] += gf[a] * w;
      o[11 + a] += (gf[a] - gi[a]) * (gf[a] - gi[a]) * w;
      o[14 + a] += gf[a] * gf[a] * w;
    }
  };
  for (int64_t p = 0; p < n_points; ++p)
  {
    double pos[3];
    matvec(sim.c, points + 3 * p, pos);
    double gi[3], gf[3], d8[8];
    double ei = interpolateTricubicGradient(vdw_grid, nx, ny, nz, gs.unit, pos, gi) * toK;
    for (int a = 0; a < 3; ++a) gi[a] *= toK;
    tricubicFractional(0, ff, gs.super, pos, probe_type, gs.unit, gs.atoms.data(), static_cast<int>(gs.atoms.size()),
                       d8);
    const double ef = d8[0] * toK;
    for (int a = 0; a < 3; ++a)
      gf[a] = (gs.unit.ic[a][0] * d8[1] + gs.unit.ic[a][1] * d8[2] + gs.unit.ic[a][2] * d8[3]) * toK;
    const double w = std::exp(-weight_beta * ef);
    accumulate(out, w, ei, ef, gi, gf);
    out[34] += 1.0;
    if (ewald_grid && probe_charge != 0.0 && ef < ff->overlap_criteria)
    {
      double ci[3], cf[3];
      const double eci = interpolateTricubicGradient(ewald_grid, nx, ny, nz, gs.unit, pos, ci) * probe_charge * toK;
      for (int a = 0; a < 3; ++a) ci[a] *= probe_charge * toK;
      tricubicFractional(1, ff, gs.super, pos, 0, gs.unit, gs.atoms.data(), static_cast<int>(gs.atoms.size()), d8);
      const double ecf = d8[0] * probe_charge * toK;
      for (int a = 0; a < 3; ++a)
        cf[a] = (gs.unit.ic[a][0] * d8[1] + gs.unit.ic[a][1] * d8[2] + gs.unit.ic[a][2] * d8[3]) * probe_charge * toK;
      accumulate(out + 17, w, eci, ecf, ci, cf);
      out[35] += 1.0;
    }
  }
}

void oracle_grid_validate_triquintic(const off* ff, const obox* unit_box, const oatom* unit_atoms, int n_unit,
                                     const obox* simulation_box, int probe_type, int nx, int ny, int nz,
                                     const double* vdw_grid, const double* ewald_grid, double probe_charge,
                                     double weight_beta, const double* points, int64_t n_points, double* out)
{
  // The grid test of the triquintic scheme (system_interpolation_grids.cpp:272-651): energy, gradient and Hessian,
  // interpolated (interpolateHessian) and analytical (calculateTriquinticFractionalAtPosition, the gradient from its
  // channels 1-3 and the Hessian from channels 4-9 mapped with the inverse cell), in K, Boltzmann-weighted. The
  // analytical channels are the exact ones (for a rectangular cell the reference's own branch scales its y and z first
  // derivatives by cell[0][0]). out: the 36 values of oracle_grid_validate, then 24 VDW and 24 charge Hessian sums
  // (interpolated, full, squared difference, squared full; components xx, xy, xz, yy, yz, zz).
  const GridSetup gs = gridSetup(unit_box, unit_atoms, n_unit, ff->cutoff_framework_vdw, nx, ny, nz);
  const Box sim = makeBox(simulation_box);
  const double toK = energyConversionFactor() * kAvogadroConstant / kMolarGasConstant;
  for (int i = 0; i < 84; ++i) out[i] = 0.0;
  auto accumulate = [&](double* o, double* oh, double w, double ei, double ef, const double* gi, const double* gf,
                        const double* hi, const double* hf)
  {
    o[0] += w;
    o[1] += ei * w;
    o[2] += ef * w;
    o[3] += (ef - ei) * (ef - ei) * w;
    o[4] += ef * ef * w;
    for (int a = 0; a < 3; ++a)
    {
      o[5 + a] += gi[a] * w;
      o[8 + a] += gf[a] * w;
      o[11 + a] += (gf[a] - gi[a]) * (gf[a] - gi[a]) * w;
      o[14 + a] += gf[a] * gf[a] * w;
    }
    for (int q = 0; q < 6; ++q)
    {
      oh[q] += hi[q] * w;
      oh[6 + q] += hf[q] * w;
      oh[12 + q] += (hf[q] - hi[q]) * (hf[q] - hi[q]) * w;
      oh[18 + q] += hf[q] * hf[q] * w;
    }
  };
  // analytical energy, gradient and Hessian from the 27 fractional channels
  auto analytical = [&](int grid_type, int type, const double* pos, double scale, double& e, double* g, double* h)
  {
    double d[27];
    triquinticFractional(grid_type, ff, gs.super, pos, type, gs.unit, gs.atoms.data(),
                         static_cast<int>(gs.atoms.size()), false, d);
    const double gfrac[3] = {d[1], d[2], d[3]};
    const double hfrac[6] = {d[4], d[5], d[6], d[7], d[8], d[9]};
    toCartesian(gs.unit, gfrac, hfrac, g, h);
    e = d[0] * scale;
    for (int a = 0; a < 3; ++a) g[a] *= scale;
    for (int q = 0; q < 6; ++q) h[q] *= scale;
  };
  for (int64_t p = 0; p < n_points; ++p)
  {
    double pos[3];
    matvec(sim.c, points + 3 * p, pos);
    double gi[3], hi[6], ef, gf[3], hf[6];
    const double ei = interpolateTriquinticHessian(vdw_grid, nx, ny, nz, gs.unit, pos, gi, hi) * toK;
    for (int a = 0; a < 3; ++a) gi[a] *= toK;
    for (int q = 0; q < 6; ++q) hi[q] *= toK;
    analytical(0, probe_type, pos, toK, ef, gf, hf);
    const double w = std::exp(-weight_beta * ef);
    accumulate(out, out + 36, w, ei, ef, gi, gf, hi, hf);
    out[34] += 1.0;
    if (ewald_grid && probe_charge != 0.0 && ef < ff->overlap_criteria)
    {
      const double sc = probe_charge * toK;
      double ci[3], chi[6], ecf, cf[3], chf[6];
      const double eci = interpolateTriquinticHessian(ewald_grid, nx, ny, nz, gs.unit, pos, ci, chi) * sc;
      for (int a = 0; a < 3; ++a) ci[a] *= sc;
      for (int q = 0; q < 6; ++q) chi[q] *= sc;
      analytical(1, 0, pos, sc, ecf, cf, chf);
      accumulate(out + 17, out + 60, w, eci, ecf, ci, cf, chi, chf);
      out[35] += 1.0;
    }
  }
}

void oracle_pair_vdw(const off* ff, double scaling_a, double scaling_b, double rr, int type_a, int type_b,
                     double out[2])
{
  pairVDW(ff, scaling_a, scaling_b, rr, type_a, type_b, out);
}

void oracle_pair_coulomb(const off* ff, double scaling_a, double scaling_b, double r, double qa, double qb,
                         double out[2])
{
  pairCoulomb(ff, scaling_a, scaling_b, r, qa, qb, out);
}

int oracle_cbmc_framework_molecule(const off* ff, const obox* box, const double* const* grids, int gnx, int gny,
                                   int gnz, const obox* grid_box, const oatom* fw, int n_fw, double cutoff_vdw,
                                   double cutoff_coulomb, const oatom* atoms, int n_atoms, int skip, oenergy* e)
{
  // cbmc/interactions_framework_molecule.cpp:31-104 (serial variant)
  std::memset(e, 0, sizeof(oenergy));
  Box b = makeBox(box);
  Box gb = grid_box ? makeBox(grid_box) : b;
  const bool useCharge = ff->use_charge != 0;
  const double overlap = ff->overlap_criteria;
  const double rcv2 = cutoff_vdw * cutoff_vdw;
  const double rcc2 = cutoff_coulomb * cutoff_coulomb;
  for (int index = 0; index < n_atoms; ++index)
  {
    if (index == skip) continue;
    const oatom& B = atoms[index];
    double posB[3] = {B.x, B.y, B.z};
    if (grids && grids[B.type] && !fractionalOf(B))
    {
      double energy = interpolateTricubic(grids[B.type], gnx, gny, gnz, gb, posB);
      if (energy > overlap) return 0;
      e->framework_molecule_vdw += energy;
      if (useCharge && grids[ff->n_types])
        e->framework_molecule_charge += B.charge * interpolateTricubic(grids[ff->n_types], gnx, gny, gnz, gb, posB);
      continue;
    }
    for (int a = 0; a < n_fw; ++a)
    {
      const oatom& A = fw[a];
      double dr[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
      pbc(b, dr);
      double rr = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
      if (rr < rcv2)
      {
        double f[2];
        pairVDW(ff, A.scaling_vdw, B.scaling_vdw, rr, A.type, B.type, f);
        if (f[0] > overlap) return 0;
        e->framework_molecule_vdw += f[0];
        addDud(e->dudlambda_vdw, groupOf(A), groupOf(B), A.scaling_vdw, B.scaling_vdw, f[1]);
      }
      if (useCharge && rr < rcc2)
      {
        double r = std::sqrt(rr);
        double f[2];
        pairCoulomb(ff, A.scaling_coulomb, B.scaling_coulomb, r, A.charge, B.charge, f);
        e->framework_molecule_charge += f[0];
        addDud(e->dudlambda_charge, groupOf(A), groupOf(B), A.scaling_coulomb, B.scaling_coulomb, f[1]);
      }
    }
  }
  return 1;
}

int oracle_cbmc_intermolecular(const off* ff, const obox* box, const oatom* molecule_atoms, int n_mol,
                               double cutoff_vdw, double cutoff_coulomb, const oatom* atoms, int n_atoms, int skip,
                               int64_t skip_background_molecule, oenergy* e)
{
  // cbmc/interactions_intermolecular.cpp:22-95
  std::memset(e, 0, sizeof(oenergy));
  Box b = makeBox(box);
  const bool useCharge = ff->use_charge != 0;
  const double overlap = ff->overlap_criteria;
  const double rcv2 = cutoff_vdw * cutoff_vdw;
  const double rcc2 = cutoff_coulomb * cutoff_coulomb;
  for (int m = 0; m < n_mol; ++m)
  {
    const oatom& A = molecule_atoms[m];
    if (skip_background_molecule >= 0 && A.molecule_id == static_cast<uint64_t>(skip_background_molecule)) continue;
    for (int index = 0; index < n_atoms; ++index)
    {
      if (index == skip) continue;
      const oatom& B = atoms[index];
      if (A.molecule_id == B.molecule_id) continue;
      double dr[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
      pbc(b, dr);
      double rr = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
      if (rr < rcv2)
      {
        double f[2];
        pairVDW(ff, A.scaling_vdw, B.scaling_vdw, rr, A.type, B.type, f);
        if (f[0] > overlap) return 0;
        e->molecule_molecule_vdw += f[0];
        addDud(e->dudlambda_vdw, groupOf(A), groupOf(B), A.scaling_vdw, B.scaling_vdw, f[1]);
      }
      if (useCharge && rr < rcc2)
      {
        double r = std::sqrt(rr);
        double f[2];
        pairCoulomb(ff, A.scaling_coulomb, B.scaling_coulomb, r, A.charge, B.charge, f);
        e->molecule_molecule_charge += f[0];
        addDud(e->dudlambda_charge, groupOf(A), groupOf(B), A.scaling_coulomb, B.scaling_coulomb, f[1]);
      }
    }
  }
  return 1;
}

int oracle_framework_molecule_energy_difference(const off* ff, const obox* box, const double* const* grids, int gnx,
                                                int gny, int gnz, const obox* grid_box, const oatom* fw, int n_fw,
                                                int charge_method_ewald, const oatom* new_atoms, int n_new,
                                                const oatom* old_atoms, int n_old, oenergy* e)
{
  // Interactions::computeFrameworkMoleculeEnergyDifference (interactions/framework_molecule.cpp:117-252): the grid
  // branch only for non-fractional atoms with a grid under the Ewald charge method; overlap (nullopt, return 0) checked
  // for the new atoms only; the result is E(new) - E(old).
  std::memset(e, 0, sizeof(oenergy));
  Box b = makeBox(box);
  Box gb = grid_box ? makeBox(grid_box) : b;
  const bool useCharge = ff->use_charge != 0;
  const double overlap = ff->overlap_criteria;
  const double rcv2 = ff->cutoff_framework_vdw * ff->cutoff_framework_vdw;
  const double rcc2 = ff->cutoff_coulomb * ff->cutoff_coulomb;
  for (int pass = 0; pass < 2; ++pass)
  {
    const oatom* atoms = pass == 0 ? new_atoms : old_atoms;
    const int n = pass == 0 ? n_new : n_old;
    const double sign = pass == 0 ? 1.0 : -1.0;
    for (int index = 0; index < n; ++index)
    {
      const oatom& B = atoms[index];
      double posB[3] = {B.x, B.y, B.z};
      if (grids && grids[B.type] && !fractionalOf(B) && charge_method_ewald)
      {
        double energy = interpolateTricubic(grids[B.type], gnx, gny, gnz, gb, posB);
        if (pass == 0 && energy > overlap) return 0;
        e->framework_molecule_vdw += sign * energy;
        if (useCharge && grids[ff->n_types])
          e->framework_molecule_charge +=
              sign * B.charge * interpolateTricubic(grids[ff->n_types], gnx, gny, gnz, gb, posB);
        continue;
      }
      for (int a = 0; a < n_fw; ++a)
      {
        const oatom& A = fw[a];
        double dr[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
        pbc(b, dr);
        double rr = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        if (rr < rcv2)
        {
          double f[2];
          pairVDW(ff, A.scaling_vdw, B.scaling_vdw, rr, A.type, B.type, f);
          if (pass == 0 && f[0] > overlap) return 0;
          e->framework_molecule_vdw += sign * f[0];
          addDud(e->dudlambda_vdw, groupOf(A), groupOf(B), A.scaling_vdw, B.scaling_vdw, sign * f[1]);
        }
        if (useCharge && rr < rcc2)
        {
          double r = std::sqrt(rr);
          double f[2];
          pairCoulomb(ff, A.scaling_coulomb, B.scaling_coulomb, r, A.charge, B.charge, f);
          e->framework_molecule_charge += sign * f[0];
          addDud(e->dudlambda_charge, groupOf(A), groupOf(B), A.scaling_coulomb, B.scaling_coulomb, sign * f[1]);
        }
      }
    }
  }
  return 1;
}

int oracle_intermolecular_energy_difference(const off* ff, const obox* box, const oatom* molecule_atoms, int n_mol,
                                            const oatom* new_atoms, int n_new, const oatom* old_atoms, int n_old,
                                            oenergy* e)
{
  // Interactions::computeInterMolecularEnergyDifference (interactions/intermolecular.cpp:198-290): every stored
  // adsorbate atom of another molecule against the new atoms (overlap checked) and the old atoms (subtracted).
  std::memset(e, 0, sizeof(oenergy));
  if (ff->omit_inter) return 1;
  Box b = makeBox(box);
  const bool useCharge = ff->use_charge != 0;
  const double overlap = ff->overlap_criteria;
  const double rcv2 = ff->cutoff_molecule_vdw * ff->cutoff_molecule_vdw;
  const double rcc2 = ff->cutoff_coulomb * ff->cutoff_coulomb;
  for (int m = 0; m < n_mol; ++m)
  {
    const oatom& A = molecule_atoms[m];
    for (int pass = 0; pass < 2; ++pass)
    {
      const oatom* atoms = pass == 0 ? new_atoms : old_atoms;
      const int n = pass == 0 ? n_new : n_old;
      const double sign = pass == 0 ? 1.0 : -1.0;
      for (int index = 0; index < n; ++index)
      {
        const oatom& B = atoms[index];
        if (A.molecule_id == B.molecule_id) continue;
        double dr[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
        pbc(b, dr);
        double rr = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        if (rr < rcv2)
        {
          double f[2];
          pairVDW(ff, A.scaling_vdw, B.scaling_vdw, rr, A.type, B.type, f);
          if (pass == 0 && f[0] > overlap) return 0;
          e->molecule_molecule_vdw += sign * f[0];
          addDud(e->dudlambda_vdw, groupOf(A), groupOf(B), A.scaling_vdw, B.scaling_vdw, sign * f[1]);
        }
        if (useCharge && rr < rcc2)
        {
          double r = std::sqrt(rr);
          double f[2];
          pairCoulomb(ff, A.scaling_coulomb, B.scaling_coulomb, r, A.charge, B.charge, f);
          e->molecule_molecule_charge += sign * f[0];
          addDud(e->dudlambda_charge, groupOf(A), groupOf(B), A.scaling_coulomb, B.scaling_coulomb, sign * f[1]);
        }
      }
    }
  }
  return 1;
}

int oracle_inside_blocked_pockets(const obox* unit_box, const double* pockets, int n_pockets, const oatom* atoms,
                                  int n_atoms)
{
  // CBMC::insideBlockedPockets (cbmc/interactions.cpp:25-52): pocket centres are fractions of the framework's unit
  // cell, the minimum image is taken in that unit cell, and the radius is scaled by the atom's VDW scaling.
  Box b = makeBox(unit_box);
  for (int i = 0; i < n_pockets; ++i)
  {
    const double radius_squared = pockets[4 * i + 3] * pockets[4 * i + 3];
    const double f[3] = {pockets[4 * i], pockets[4 * i + 1], pockets[4 * i + 2]};
    double pos[3];
    matvec(b.c, f, pos);
    for (int a = 0; a < n_atoms; ++a)
    {
      double dr[3] = {atoms[a].x - pos[0], atoms[a].y - pos[1], atoms[a].z - pos[2]};
      pbc(b, dr);
      if (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2] < atoms[a].scaling_vdw * radius_squared) return 1;
    }
  }
  return 0;
}

int oracle_external_field_energy(int surface_type, const double* geometry, const obox* box, const double* grid,
                                 int gnx, int gny, int gnz, const obox* grid_box, const oatom* atoms, int n_atoms,
                                 int skip, double* energy)
{
  // CBMC::computeExternalFieldEnergy (cbmc/interactions_external_field.cpp:22-200): a grid (scaled by the atom's VDW
  // scaling) takes precedence; otherwise the analytic surfaces of the switch, the confinements returning nullopt
  // (here 0) outside; every other surface type adds nothing.
  *energy = 0.0;
  Box b = makeBox(box);
  Box gb = grid_box ? makeBox(grid_box) : b;
  for (int index = 0; index < n_atoms; ++index)
  {
    if (index == skip) continue;
    const oatom& A = atoms[index];
    const double pos[3] = {A.x, A.y, A.z};
    double e = 0.0;
    if (grid)
      e = A.scaling_vdw * interpolateTricubic(grid, gnx, gny, gnz, gb, pos);
    else if (surface_type == 8)  // MullerBrown
    {
      const double Ak[4] = {-200.0, -100.0, -170.0, -15.0}, ak[4] = {-1.0, -1.0, -6.5, -0.7},
                   x0[4] = {1.0, 0.0, -0.5, -1.0}, bk[4] = {0.0, 0.0, 11.0, 0.6}, y0[4] = {0.0, 0.5, 1.5, 1.0},
                   ck[4] = {-10.0, -10.0, -6.5, 0.7};
      for (int i = 0; i < 4; ++i)
        e += Ak[i] * std::exp(ak[i] * (pos[0] - x0[i]) * (pos[0] - x0[i]) +
                              bk[i] * (pos[0] - x0[i]) * (pos[1] - y0[i]) + ck[i] * (pos[1] - y0[i]) * (pos[1] - y0[i]));
    }
    else if (surface_type == 3)  // ThirdOrderPolynomialTestFunction
      e = pos[0] * pos[1] * pos[2];
    else if (surface_type >= 11 && surface_type <= 16)  // CylinderX/Y/Z, RectangleX/Y/Z
    {
      const int axis = (surface_type - 11) % 3;
      double fb[3] = {0.5, 0.5, 0.5}, fe[3] = {0.5, 0.5, 0.5};
      fb[axis] = 0.0;
      fe[axis] = 1.0;
      double cb[3], ce[3];
      matvec(b.c, fb, cb);
      matvec(b.c, fe, ce);
      double v[3] = {ce[0] - cb[0], ce[1] - cb[1], ce[2] - cb[2]};
      const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      for (double& x : v) x /= len;
      const double d[3] = {pos[0] - cb[0], pos[1] - cb[1], pos[2] - cb[2]};
      const double w[3] = {d[1] * v[2] - d[2] * v[1], d[2] * v[0] - d[0] * v[2], d[0] * v[1] - d[1] * v[0]};
      bool inside;
      if (surface_type <= 13)
        inside = w[0] * w[0] + w[1] * w[1] + w[2] * w[2] < geometry[0] * geometry[0];
      else if (surface_type == 14)
        inside = std::fabs(w[1]) < geometry[0] && std::fabs(w[2]) < geometry[1];
      else if (surface_type == 15)
        inside = std::fabs(w[2]) < geometry[0] && std::fabs(w[0]) < geometry[1];
      else
        inside = std::fabs(w[1]) < geometry[0] && std::fabs(w[0]) < geometry[1];
      if (!inside) return 0;
    }
    *energy += e;
  }
  return 1;
}

int64_t oracle_ewald_kvectors(const off* ff, const obox* box, int32_t* kvec, double* temp, double* single_ion_sum)
{
  Box b = makeBox(box);
  const double alpha_squared = ff->ewald_alpha * ff->ewald_alpha;
  int64_t n = 0;
  double sum = 0.0;
  forEachK(ff, b,
           [&](int kx, int ky, int kz, double rksq, double factor)
           {
             double t = factor * std::exp((-0.25 / alpha_squared) * rksq) / rksq;
             if (kvec)
             {
               kvec[3 * n + 0] = kx;
               kvec[3 * n + 1] = ky;
               kvec[3 * n + 2] = kz;
             }
             if (temp) temp[n] = t;
             sum += t;
             ++n;
           });
  if (single_ion_sum) *single_ion_sum = sum;
  return n;
}

double oracle_ewald_delta_parallel(const off* ff, const obox* box, const int32_t* kvec, const double* temp, int64_t nk,
                                   const double* stored, const oatom* new_atoms, int n_new, const oatom* old_atoms,
                                   int n_old, double* trial, int threads)
{
  // The k loop of energyDifferenceEwaldFourier (ewald.cpp:1098-1162) without dU/dlambda groups, over a precomputed
  // k table (oracle_ewald_kvectors), parallelised over k with OpenMP: the CPU baseline on all host cores. Returns the
  // Fourier energy change; trial (10 doubles per k, groups zero) receives the trial structure factors.
  Box b = makeBox(box);
  const int n = n_new + n_old;
  std::vector<const oatom*> ptr(n);
  for (int i = 0; i < n_old; ++i) ptr[i] = &old_atoms[i];
  for (int i = 0; i < n_new; ++i) ptr[n_old + i] = &new_atoms[i];
  EikTables eik(b, ptr, ff->kmax_x, ff->kmax_y, ff->kmax_z);
  std::vector<double> w(n);
  for (int i = 0; i < n; ++i) w[i] = (i < n_old ? -1.0 : 1.0) * ptr[i]->scaling_coulomb * ptr[i]->charge;
  double energy = 0.0;
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) reduction(+ : energy) num_threads(threads)
#endif
  for (int64_t k = 0; k < nk; ++k)
  {
    const int kx = kvec[3 * k], ky = kvec[3 * k + 1], kz = kvec[3 * k + 2];
    Cplx d{0.0, 0.0};
    for (int i = 0; i < n; ++i)
    {
      const Cplx ei = cmul(eik.xy(i, kx, ky), eik.zf(i, kz));
      d.re += w[i] * ei.re;
      d.im += w[i] * ei.im;
    }
    const double* s = stored + 10 * k;
    const Cplx S{s[0], s[1]};
    const Cplx T{S.re + d.re, S.im + d.im};
    energy += temp[k] * (norm2(T) - norm2(S));
    if (trial)
    {
      double* t = trial + 10 * k;
      t[0] = T.re;
      t[1] = T.im;
      for (int g = 2; g < 10; ++g) t[g] = 0.0;
    }
  }
  (void)threads;
  return energy;
}

void oracle_ewald_rigid(const off* ff, const obox* box, const oatom* fw, int n_fw, double* s_rigid)
{
  // precomputeEwaldFourierRigid, ewald.cpp:276-348
  Box b = makeBox(box);
  std::vector<const oatom*> ptr(n_fw);
  for (int i = 0; i < n_fw; ++i) ptr[i] = &fw[i];
  EikTables eik(b, ptr, ff->kmax_x, ff->kmax_y, ff->kmax_z);
  int64_t nvec = 0;
  int lastKx = -1, lastKy = 1 << 30;
  std::vector<Cplx> xy(n_fw);
  forEachK(ff, b,
           [&](int kx, int ky, int kz, double, double)
           {
             if (kx != lastKx || ky != lastKy)
             {
               for (int i = 0; i < n_fw; ++i) xy[i] = eik.xy(i, kx, ky);
               lastKx = kx;
               lastKy = ky;
             }
             Cplx sum{0.0, 0.0};
             for (int i = 0; i < n_fw; ++i)
             {
               Cplx e = cmul(xy[i], eik.zf(i, kz));
               double w = fw[i].scaling_coulomb * fw[i].charge;
               sum.re += w * e.re;
               sum.im += w * e.im;
             }
             s_rigid[2 * nvec] = sum.re;
             s_rigid[2 * nvec + 1] = sum.im;
             ++nvec;
           });
}

void oracle_ewald_fourier_energy(const off* ff, const obox* box, const double* s_rigid, const oatom* atoms, int n,
                                 const int32_t* molecule_sizes, int n_molecules, double net_charge_framework,
                                 double* stored, oenergy* e)
{
  // computeEwaldFourierEnergy, ewald.cpp:352-563 (Ewald charge method)
  std::memset(e, 0, sizeof(oenergy));
  if (!ff->use_charge) return;
  Box b = makeBox(box);
  const double alpha = ff->ewald_alpha;
  const double alpha_squared = alpha * alpha;
  const double C = coulombFactor();
  std::vector<const oatom*> ptr(n);
  for (int i = 0; i < n; ++i) ptr[i] = &atoms[i];
  EikTables eik(b, ptr, ff->kmax_x, ff->kmax_y, ff->kmax_z);
  double singleIonFourierSum = 0.0;
  int64_t nvec = 0;
  int lastKx = -1, lastKy = 1 << 30;
  std::vector<Cplx> xy(n);
  forEachK(ff, b,
           [&](int kx, int ky, int kz, double rksq, double factor)
           {
             if (kx != lastKx || ky != lastKy)
             {
               for (int i = 0; i < n; ++i) xy[i] = eik.xy(i, kx, ky);
               lastKx = kx;
               lastKy = ky;
             }
             double temp = factor * std::exp((-0.25 / alpha_squared) * rksq) / rksq;
             singleIonFourierSum += temp;
             Cplx ck{0.0, 0.0};
             Cplx cg[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
             for (int i = 0; i < n; ++i)
             {
               Cplx ei = cmul(xy[i], eik.zf(i, kz));
               double q = atoms[i].charge, sc = atoms[i].scaling_coulomb;
               ck.re += sc * q * ei.re;
               ck.im += sc * q * ei.im;
               int g = groupOf(atoms[i]);
               if (g != 0)
               {
                 cg[g - 1].re += q * ei.re;
                 cg[g - 1].im += q * ei.im;
               }
             }
             Cplx rigid{0.0, 0.0};
             if (s_rigid) rigid = Cplx{s_rigid[2 * nvec], s_rigid[2 * nvec + 1]};
             Cplx rigidG[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
             Cplx total{rigid.re + ck.re, rigid.im + ck.im};
             Cplx totalG[4];
             for (int g = 0; g < 4; ++g) totalG[g] = Cplx{rigidG[g].re + cg[g].re, rigidG[g].im + cg[g].im};
             double rigidEnergy = temp * (rigid.re * rigid.re + rigid.im * rigid.im);
             e->ewald_fourier += temp * (total.re * total.re + total.im * total.im) - rigidEnergy;
             if (ff->omit_inter) e->ewald_fourier -= temp * (ck.re * ck.re + ck.im * ck.im);
             addFourierDUdlambda(e, 2.0 * temp, total, totalG);
             addFourierDUdlambda(e, -2.0 * temp, rigid, rigidG);
             if (stored)
             {
               double* s = stored + 10 * nvec;
               s[0] = total.re;
               s[1] = total.im;
               for (int g = 0; g < 4; ++g)
               {
                 s[2 + 2 * g] = totalG[g].re;
                 s[3 + 2 * g] = totalG[g].im;
               }
             }
             ++nvec;
           });
  if (!ff->omit_inter)
  {
    double prefactor_self = C * alpha / std::sqrt(kPi);
    for (int i = 0; i < n; ++i)
    {
      double q = atoms[i].charge, sc = atoms[i].scaling_coulomb;
      int g = groupOf(atoms[i]);
      e->ewald_self -= prefactor_self * sc * q * sc * q;
      if (g != 0) e->dudlambda_ewald[g - 1] -= 2.0 * prefactor_self * sc * q * q;
    }
    int index = 0;
    for (int m = 0; m < n_molecules; ++m)
    {
      int size = molecule_sizes[m];
      const oatom* span = atoms + index;
      for (int i = 0; i + 1 < size; ++i)
        for (int j = i + 1; j < size; ++j)
        {
          double dr[3] = {span[i].x - span[j].x, span[i].y - span[j].y, span[i].z - span[j].z};
          pbc(b, dr);
          double r = std::sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
          double sA = span[i].scaling_coulomb, sB = span[j].scaling_coulomb;
          double pot, dudl;
          exclusionFactors(alpha, sA * sB, r, pot, dudl);
          double prefactor = C * span[i].charge * span[j].charge;
          e->ewald_exclusion -= sA * sB * prefactor * pot;
          addDud(e->dudlambda_ewald, groupOf(span[i]), groupOf(span[j]), sA, sB, -prefactor * dudl);
        }
      index += size;
    }
  }
  // net-charge correction (ewald.cpp:526-560)
  double netChargeAdsorbates = 0.0;
  double netChargeDerivative[4] = {0, 0, 0, 0};
  for (int i = 0; i < n; ++i)
  {
    netChargeAdsorbates += atoms[i].scaling_coulomb * atoms[i].charge;
    int g = groupOf(atoms[i]);
    if (g != 0) netChargeDerivative[g - 1] += atoms[i].charge;
  }
  double uIon = -(singleIonFourierSum - C * alpha / std::sqrt(kPi));
  if (ff->omit_inter)
  {
    e->ewald_fourier += 2.0 * uIon * net_charge_framework * netChargeAdsorbates;
    for (int g = 0; g < 4; ++g) e->dudlambda_ewald[g] += 2.0 * uIon * net_charge_framework * netChargeDerivative[g];
  }
  else
  {
    e->ewald_fourier += uIon * (2.0 * net_charge_framework + netChargeAdsorbates) * netChargeAdsorbates;
    for (int g = 0; g < 4; ++g)
      e->dudlambda_ewald[g] += 2.0 * uIon * (net_charge_framework + netChargeAdsorbates) * netChargeDerivative[g];
  }
}

void oracle_ewald_delta(const off* ff, const obox* box, const double* stored, const oatom* new_atoms, int n_new,
                        const oatom* old_atoms, int n_old, double net_charge, const double* net_charge_derivative_ext,
                        double* trial, oenergy* e)
{
  // energyDifferenceEwaldFourier, ewald.cpp:1043-1244 (Ewald charge method)
  std::memset(e, 0, sizeof(oenergy));
  if (!ff->use_charge) return;
  Box b = makeBox(box);
  const double alpha = ff->ewald_alpha;
  const double alpha_squared = alpha * alpha;
  const double C = coulombFactor();
  const int n = n_new + n_old;
  std::vector<const oatom*> ptr(n);  // old atoms first, then new (ewald_kvector.ixx buildEikTables overload)
  for (int i = 0; i < n_old; ++i) ptr[i] = &old_atoms[i];
  for (int i = 0; i < n_new; ++i) ptr[n_old + i] = &new_atoms[i];
  EikTables eik(b, ptr, ff->kmax_x, ff->kmax_y, ff->kmax_z);
  double singleIonFourierSum = 0.0;
  int64_t nvec = 0;
  int lastKx = -1, lastKy = 1 << 30;
  std::vector<Cplx> xy(n);
  forEachK(ff, b,
           [&](int kx, int ky, int kz, double rksq, double factor)
           {
             if (kx != lastKx || ky != lastKy)
             {
               for (int i = 0; i < n; ++i) xy[i] = eik.xy(i, kx, ky);
               lastKx = kx;
               lastKy = ky;
             }
             Cplx co{0, 0}, cn{0, 0};
             Cplx go[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}}, gn[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
             for (int i = 0; i < n; ++i)
             {
               Cplx ei = cmul(xy[i], eik.zf(i, kz));
               const oatom& A = *ptr[i];
               double q = A.charge, sc = A.scaling_coulomb;
               Cplx& c = (i < n_old) ? co : cn;
               Cplx* g = (i < n_old) ? go : gn;
               c.re += sc * q * ei.re;
               c.im += sc * q * ei.im;
               int gi = groupOf(A);
               if (gi != 0)
               {
                 g[gi - 1].re += q * ei.re;
                 g[gi - 1].im += q * ei.im;
               }
             }
             double temp = factor * std::exp((-0.25 / alpha_squared) * rksq) / rksq;
             singleIonFourierSum += temp;
             const double* s = stored + 10 * nvec;
             Cplx S{s[0], s[1]};
             Cplx SG[4];
             for (int g = 0; g < 4; ++g) SG[g] = Cplx{s[2 + 2 * g], s[3 + 2 * g]};
             Cplx T{S.re + cn.re - co.re, S.im + cn.im - co.im};
             Cplx TG[4];
             for (int g = 0; g < 4; ++g) TG[g] = Cplx{SG[g].re + gn[g].re - go[g].re, SG[g].im + gn[g].im - go[g].im};
             e->ewald_fourier += temp * norm2(T);
             e->ewald_fourier -= temp * norm2(S);
             addFourierDUdlambda(e, 2.0 * temp, T, TG);
             addFourierDUdlambda(e, -2.0 * temp, S, SG);
             if (trial)
             {
               double* t = trial + 10 * nvec;
               t[0] = T.re;
               t[1] = T.im;
               for (int g = 0; g < 4; ++g)
               {
                 t[2 + 2 * g] = TG[g].re;
                 t[3 + 2 * g] = TG[g].im;
               }
             }
             ++nvec;
           });
  // intramolecular exclusion, ewald.cpp:1164-1219
  auto exclusion = [&](const oatom* atoms, int count, double sign)
  {
    for (int i = 0; i < count; ++i)
      for (int j = i + 1; j < count; ++j)
      {
        if (atoms[i].molecule_id != atoms[j].molecule_id) continue;
        double dr[3] = {atoms[i].x - atoms[j].x, atoms[i].y - atoms[j].y, atoms[i].z - atoms[j].z};
        pbc(b, dr);
        double r = std::sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        double sA = atoms[i].scaling_coulomb, sB = atoms[j].scaling_coulomb;
        double pot, dudl;
        exclusionFactors(alpha, sA * sB, r, pot, dudl);
        double prefactor = C * atoms[i].charge * atoms[j].charge;
        e->ewald_exclusion += sign * sA * sB * prefactor * pot;
        addDud(e->dudlambda_ewald, groupOf(atoms[i]), groupOf(atoms[j]), sA, sB, sign * prefactor * dudl);
      }
  };
  exclusion(old_atoms, n_old, 1.0);
  exclusion(new_atoms, n_new, -1.0);
  // self energy, ewald.cpp:1221-1238
  double prefactor_self = C * ff->ewald_alpha / std::sqrt(kPi);
  for (int i = 0; i < n_old; ++i)
  {
    double q = old_atoms[i].charge, sc = old_atoms[i].scaling_coulomb;
    int g = groupOf(old_atoms[i]);
    e->ewald_self += prefactor_self * sc * q * sc * q;
    if (g != 0) e->dudlambda_ewald[g - 1] += 2.0 * prefactor_self * sc * q * q;
  }
  for (int i = 0; i < n_new; ++i)
  {
    double q = new_atoms[i].charge, sc = new_atoms[i].scaling_coulomb;
    int g = groupOf(new_atoms[i]);
    e->ewald_self -= prefactor_self * sc * q * sc * q;
    if (g != 0) e->dudlambda_ewald[g - 1] -= 2.0 * prefactor_self * sc * q * q;
  }
  // net-charge correction difference, ewald.cpp:181-208
  double deltaCharge = 0.0;
  double dNew[4], dOld[4];
  for (int g = 0; g < 4; ++g) dNew[g] = dOld[g] = net_charge_derivative_ext ? net_charge_derivative_ext[g] : 0.0;
  for (int i = 0; i < n_old; ++i)
  {
    deltaCharge -= old_atoms[i].scaling_coulomb * old_atoms[i].charge;
    int g = groupOf(old_atoms[i]);
    if (g != 0) dOld[g - 1] += old_atoms[i].charge;
  }
  for (int i = 0; i < n_new; ++i)
  {
    deltaCharge += new_atoms[i].scaling_coulomb * new_atoms[i].charge;
    int g = groupOf(new_atoms[i]);
    if (g != 0) dNew[g - 1] += new_atoms[i].charge;
  }
  double uIon = -(singleIonFourierSum - C * alpha / std::sqrt(kPi));
  double netChargeNew = net_charge + deltaCharge;
  e->ewald_fourier += uIon * (netChargeNew * netChargeNew - net_charge * net_charge);
  for (int g = 0; g < 4; ++g)
    e->dudlambda_ewald[g] += 2.0 * uIon * (netChargeNew * dNew[g] - net_charge * dOld[g]);
}

double oracle_ewald_single_ion(const off* ff, const obox* box, const double* pos, double charge)
{
  // computeEwaldFourierEnergySingleIon, ewald.cpp:210-274
  Box b = makeBox(box);
  const double alpha = ff->ewald_alpha;
  const double alpha_squared = alpha * alpha;
  oatom a{};
  a.x = pos[0];
  a.y = pos[1];
  a.z = pos[2];
  std::vector<const oatom*> ptr{&a};
  EikTables eik(b, ptr, ff->kmax_x, ff->kmax_y, ff->kmax_z);
  double energy_sum = 0.0;
  forEachK(ff, b,
           [&](int kx, int ky, int kz, double rksq, double)
           {
             double factor = (kx == 0) ? 1.0 : 2.0;
             Cplx e = cmul(eik.xy(0, kx, ky), eik.zf(0, kz));
             Cplx ck{charge * e.re, charge * e.im};
             energy_sum += factor * norm2(ck) * std::exp((-0.25 / alpha_squared) * rksq) / rksq;
           });
  return -coulombFactor() * ((2.0 * kPi / b.volume) * energy_sum - alpha / std::sqrt(kPi));
}

int oracle_select_trial(const double* log_boltzmann, int n, double uniform)
{
  // CBMC::selectTrialPosition, cbmc/util.cpp:14-47
  double largest = log_boltzmann[0];
  for (int i = 1; i < n; ++i) largest = std::max(largest, log_boltzmann[i]);
  std::vector<double> shifted(n);
  double sum = 0.0;
  for (int i = 0; i < n; ++i)
  {
    shifted[i] = std::exp(log_boltzmann[i] - largest);
    sum += shifted[i];
  }
  int selected = 0;
  double cumw = shifted[0];
  double ws = uniform * sum;
  while (selected + 1 < n && cumw < ws) cumw += shifted[++selected];
  return selected;
}
void oracle_triquintic_fractional_at_position(int grid_type, const off* ff, const obox* super_box, const double* pos,
                                              int type_a, const obox* unit_box, const oatom* super_atoms, int n,
                                              int reference_rectangular, double out[27])
{
  Box sb = makeBox(super_box), ub = makeBox(unit_box);
  triquinticFractional(grid_type, ff, sb, pos, type_a, ub, super_atoms, n, reference_rectangular != 0, out);
}

int oracle_make_triquintic_grid(int grid_type, const off* ff, const obox* unit_box, const oatom* unit_atoms,
                                int n_unit, int probe_type, double cutoff, int nx, int ny, int nz,
                                int reference_rectangular, const int64_t* points, int64_t n_points, int threads,
                                double* out)
{
  GridSetup s = gridSetup(unit_box, unit_atoms, n_unit, cutoff, nx, ny, nz);
  const int64_t total = points ? n_points : static_cast<int64_t>(nx) * ny * nz;
#ifdef _OPENMP
  if (threads < 1) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
  for (int64_t p = 0; p < total; ++p)
  {
    const int64_t flat = points ? points[p] : p;
    const int64_t i = flat % nx, j = (flat / nx) % ny, k = flat / (static_cast<int64_t>(nx) * ny);
    double* dst = points ? out + 27 * p : out + 27 * flat;
    gridPointQuintic(grid_type, ff, s, probe_type, i, j, k, reference_rectangular != 0, dst);
  }
  (void)threads;
  return static_cast<int>(s.atoms.size());
}

double oracle_triquintic_interpolate(const double* data, int nx, int ny, int nz, const obox* unit_box,
                                     const double* pos, double* grad)
{
  Box ub = makeBox(unit_box);
  return interpolateTriquintic(data, nx, ny, nz, ub, pos, grad);
}

double oracle_interpolant_from_corners(int scheme, const double* X, const double* s, double* ds)
{
  double d[3];
  const double v = scheme == 27 ? quinticFromCorners(X, s, d) : cubicFromCorners(X, s, d);
  if (ds)
    for (int a = 0; a < 3; ++a) ds[a] = d[a];
  return v;
}

void oracle_triquintic_matrix(double* m)
{
  const auto& M = triquinticMatrix().m;
  std::memcpy(m, M.data(), sizeof(double) * M.size());
}
}

// FP32 reciprocal, reciprocal square root and erfc for the FP32 pair kernels (own code: hardware approximations
// refined by one Newton step, and erfc as exp(-x^2) times a fitted rational-in-t polynomial).
#pragma once

namespace rgd
{
// FP32 reciprocal: the hardware approximation refined by one Newton step (x (2 - a x)), ~0.5 ulp
__device__ __forceinline__ float rcpRn(float a)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  const float e = fmaf(-a, r, 1.0f);
  return fmaf(r, e, r);
}
// FP32 reciprocal square root, refined by one Newton step (r (3 - a r^2) / 2)
__device__ __forceinline__ float rsqrtRn(float a)
{
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  const float h = 0.5f * a * r;
  return r * fmaf(-h, r, 1.5f);
}
// exp(x) as 2^(x log2 e) from the hardware base-2 exponential (ex2.approx, a few ulp): the Gaussian factor of the FP32
// Ewald grid terms, whose FP32 rounding of the large cancelling pair terms already dominates the grid error
__device__ __forceinline__ float expApprox(float x)
{
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x * 1.4426950408889634f));
  return r;
}
// the hardware reciprocal and reciprocal square root unrefined (a few ulp): the FP32 grid kernels, whose error is
// dominated by the FP32 rounding of the large cancelling pair terms
__device__ __forceinline__ float rcpApprox(float a)
{
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ float rsqrtApprox(float a)
{
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
  return r;
}
// erfc(x) = exp(-x^2) R(x) for 0 <= x <= 4, with R(x) = exp(x^2) erfc(x) fitted (weighted least squares in Chebyshev
// form, relative error 4e-8 in FP64, ~2 ulp in FP32) as a degree-9 polynomial in t = 1 / (1 + x/2); the caller passes
// exp(-x^2), which the derivative factors need anyway. REFINED = false takes t from the unrefined reciprocal.
template <bool REFINED = true>
__device__ __forceinline__ float erfcFromExp(float x, float expmx2)
{
  const float t = REFINED ? rcpRn(fmaf(0.5f, x, 1.0f)) : rcpApprox(fmaf(0.5f, x, 1.0f));
  float r = -0.02496027760207653f;
  r = fmaf(r, t, 0.09420006722211838f);
  r = fmaf(r, t, -0.024484887719154358f);
  r = fmaf(r, t, -0.36430737376213074f);
  r = fmaf(r, t, 0.534475564956665f);
  r = fmaf(r, t, -0.11705945432186127f);
  r = fmaf(r, t, 0.3620023727416992f);
  r = fmaf(r, t, 0.25453805923461914f);
  r = fmaf(r, t, 0.2858136296272278f);
  r = fmaf(r, t, -0.00021772264153696597f);
  return expmx2 * r;
}
// erf(x)/x as a polynomial in u = x^2 for 0 <= x <= 2 (FP64): a Chebyshev least-squares fit of erf(sqrt(u))/sqrt(u) on
// u in [0, 4] against a 40-digit reference, in monomial form, relative error 2e-15. erf(x)/x is entire, so the
// complement erfc(x)/x = 1/x - erf(x)/x needs no exponential and no branch (relative error 4e-13 for x <= 2).
constexpr double kErfOverXMax = 2.0;
__device__ __forceinline__ double erfOverX(double u)
{
  double r = 1.805761181299233e-16;
  r = fma(r, u, -1.0300117447682573e-14);
  r = fma(r, u, 2.927836726213971e-13);
  r = fma(r, u, -5.731081299066304e-12);
  r = fma(r, u, 8.96014012256378e-11);
  r = fma(r, u, -1.2127292658512346e-09);
  r = fma(r, u, 1.4763819202890526e-08);
  r = fma(r, u, -1.635716222383698e-07);
  r = fma(r, u, 1.6460811429838825e-06);
  r = fma(r, u, -1.4925505494318574e-05);
  r = fma(r, u, 0.00012055321281183126);
  r = fma(r, u, -0.000854832635719831);
  r = fma(r, u, 0.005223977599866574);
  r = fma(r, u, -0.026866170638949895);
  r = fma(r, u, 0.11283791670871149);
  r = fma(r, u, -0.37612638903178647);
  return fma(r, u, 1.1283791670955123);
}
}  // namespace rgd

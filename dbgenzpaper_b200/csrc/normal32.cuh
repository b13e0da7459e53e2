// normal32.cuh -- FP32 normal tail mass and inverse of the mixed-precision
// step, written for this library (no dependencies: device code only).
//
//   tail_mass_f32(x) = erfc(x) / 2 = Phi(-sqrt(2) x),   0 <= x <= 9,
//
// in the form erfc(x) = t exp(P(t) - x^2), t = 1 / (1 + x/2), with P a
// degree-9 polynomial: the form of the Chebyshev-fitted complementary error
// function of Press, Teukolsky, Vetterling and Flannery (Numerical Recipes,
// "erfcc").  The coefficients here are our own: a least-squares fit of
// P(t) = ln(erfcx(x)) - ln(t) on 400,001 points of [0, 9] in double
// precision (maximum error of the fit 2.2e-7 in P).  Evaluated in FP32 with
// one reciprocal, nine FMAs and one exp2 and no branches; the relative error
// against erfc is below 3e-6 for x <= 4.5 and below 1.5e-5 up to x = 9 (the
// FP32 rounding of the exponent P - x^2 dominates there, where the mass is
// below 1e-10).
#pragma once

namespace dbgz {

// 2^z by the SFU (ex2.approx.ftz: relative error about 2^-22; results below
// 2^-126 flush to zero, -inf gives 0).
__device__ __forceinline__ float exp2_sfu(float z) {
  float e;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(z));
  return e;
}

__device__ __forceinline__ float tail_mass_f32(float x) {
  const float t = __fdividef(1.0f, fmaf(0.5f, x, 1.0f));
  float p = 1.6112529716e-01f;
  p = fmaf(p, t, -7.6098558876e-01f);
  p = fmaf(p, t, 1.3262850294e+00f);
  p = fmaf(p, t, -8.9638341094e-01f);
  p = fmaf(p, t, 6.4102997549e-02f);
  p = fmaf(p, t, -6.4260147179e-02f);
  p = fmaf(p, t, 5.3133554076e-02f);
  p = fmaf(p, t, 3.8353175424e-01f);
  p = fmaf(p, t, 9.9890822443e-01f);
  p = fmaf(p, t, -1.2654574945e+00f);
  // z = (p - x^2) log2(e) >= -117 here, so no subnormal result is flushed
  return 0.5f * t * exp2_sfu((p - x * x) * 1.4426950408889634f);
}

// Phi^-1(p) for 0 < p <= 1/2 (the smaller tail: the step forms u or 1 - u,
// whichever is below 1/2), FP32, without branches.  The form is M. Giles'
// ("Approximating the erfinv function", GPU Computing Gems Jade, 2011):
// with x = 1 - 2p and w = -ln(4 p (1 - p)) = -ln(1 - x^2),
//   erfinv(x) = x P(w - 2.5)          for w < 5   (p > 1.69e-3),
//   erfinv(x) = T(sqrt(w) - 4)        for w >= 5  (p down to 2.2e-16, w <= 34.7),
// and Phi^-1(p) = -sqrt(2) erfinv(x).  P (degree 8) and T (degree 9) are our
// own weighted least-squares fits of the relative error in double precision
// (maximum 9.4e-8 and 5.8e-8); both are evaluated and the region selected, so
// the code has no branch.  Relative error in FP32 below 4e-7 for p >= 2.2e-16.
__device__ __forceinline__ float phi_inv_lower_f32(float p) {
  const float w = -__logf(4.0f * p * (1.0f - p));
  const float x = fmaf(-2.0f, p, 1.0f);
  const float tc = w - 2.5f;
  float pc = 2.854775242e-08f;
  pc = fmaf(pc, tc, 3.437494356e-07f);
  pc = fmaf(pc, tc, -3.528993161e-06f);
  pc = fmaf(pc, tc, -4.396994196e-06f);
  pc = fmaf(pc, tc, 2.186026004e-04f);
  pc = fmaf(pc, tc, -1.253706953e-03f);
  pc = fmaf(pc, tc, -4.177708101e-03f);
  pc = fmaf(pc, tc, 2.466407258e-01f);
  pc = fmaf(pc, tc, 1.501409422e+00f);
  const float ts = w * rsqrtf(w) - 4.0f;
  float pt = 8.193106379e-07f;
  pt = fmaf(pt, ts, -1.490730122e-06f);
  pt = fmaf(pt, ts, -6.624017282e-06f);
  pt = fmaf(pt, ts, 2.765589313e-05f);
  pt = fmaf(pt, ts, -8.117484620e-05f);
  pt = fmaf(pt, ts, 2.877970689e-04f);
  pt = fmaf(pt, ts, -8.563289957e-04f);
  pt = fmaf(pt, ts, 1.256645993e-03f);
  pt = fmaf(pt, ts, 1.009495442e+00f);
  pt = fmaf(pt, ts, 3.839783388e+00f);
  return -1.41421356237f * (w < 5.0f ? pc * x : pt);
}

}  // namespace dbgz

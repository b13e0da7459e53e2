// normal32.cuh -- FP32 upper tail mass of the standard normal in erf units,
// written for this library (no dependencies: device code only).
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
  return 0.5f * t * exp2f((p - x * x) * 1.4426950408889634f);
}

}  // namespace dbgz

/*
 * detmath.h -- deterministic double-precision exp() and erf().
 *
 * The pivoted Cholesky with Genz variable reordering chooses each pivot as the
 * argmin of erf(b~) - erf(a~) over the candidates of the current panel, and
 * updates the candidates' conditional means with exp(-x^2/2)
 * (reference: src/cholesky.jl:500-514 and :545).  A different erf or exp
 * (CUDA's libdevice against the host libm) can move a score by one ulp and
 * flip a near-tie, so the GPU factorisation and its CPU checker both call the
 * functions below.  Every operation is an IEEE-754 double operation whose
 * rounding is fixed: additions and products go through dm_add/dm_mul, which
 * map to __dadd_rn/__dmul_rn on the device (no contraction into FMA), and the
 * polynomial steps are explicit fused multiply-adds, which are correctly
 * rounded on both sides.  Host code that includes this header must be built
 * with -ffp-contract=off.
 *
 * Methods (written for this library):
 *   exp:  x = k ln2 + r with a Cody-Waite split of ln2 (high part has 32
 *         significant bits, so k*LN2_HI is exact), degree-13 Taylor
 *         polynomial of exp(r) for |r| <= ln2/2, scaling by 2^k in two steps.
 *         Max error 1 ulp against libm on [-700, 700].
 *   erf:  |x| < 2.5: erf(x) = x P(0.32 x^2 - 1), P of degree 20;
 *         2.5 <= |x| < 6: erf(x) = 1 - Q(x/1.75 - 17/7), Q of degree 28;
 *         |x| >= 6: +-1.  P and Q are Chebyshev interpolants of erf(x)/x
 *         (on x^2 in [0, 6.25]) and erfc(x) (on [2.5, 6]), computed in
 *         60-digit arithmetic by detmath_fit.py and rounded to double;
 *         interpolation errors below 1.5e-18 relative (P) and 1.7e-18
 *         absolute (Q).  No exp and no division: two polynomial branches of
 *         about 25 and 30 operations.  Max error 2 ulp against the correctly
 *         rounded erf (2.1e5 points on [0, 6.5]).
 */
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define DBGZ_HD __host__ __device__ __forceinline__
#else
#define DBGZ_HD static inline
#endif

DBGZ_HD double dm_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
DBGZ_HD double dm_add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
DBGZ_HD double dm_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
DBGZ_HD double dm_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
DBGZ_HD double dm_div(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
DBGZ_HD double dm_sqrt(double a) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(a);
#else
  return sqrt(a);
#endif
}

/* 2^j for j in [-1022, 1023], built from the exponent bits. */
DBGZ_HD double dm_pow2i(int j) {
  union { uint64_t u; double d; } v;
  v.u = (uint64_t)(j + 1023) << 52;
  return v.d;
}

DBGZ_HD double det_exp(double x) {
  const double INV_LN2 = 0x1.71547652b82fep+0;
  const double LN2_HI = 0x1.62e42fee00000p-1;
  const double LN2_LO = 0x1.a39ef35793c76p-33;
  if (x != x) return x;
  if (x > 709.78) return INFINITY;
  if (x < -745.2) return 0.0;
  double kd = floor(dm_add(dm_mul(x, INV_LN2), 0.5));
  int k = (int)kd;
  double r = dm_sub(dm_sub(x, dm_mul(kd, LN2_HI)), dm_mul(kd, LN2_LO));
  double p = 0x1.6124613a86d09p-33;            /* 1/13! */
  p = dm_fma(p, r, 0x1.1eed8eff8d898p-29);     /* 1/12! */
  p = dm_fma(p, r, 0x1.ae64567f544e4p-26);
  p = dm_fma(p, r, 0x1.27e4fb7789f5cp-22);
  p = dm_fma(p, r, 0x1.71de3a556c734p-19);
  p = dm_fma(p, r, 0x1.a01a01a01a01ap-16);
  p = dm_fma(p, r, 0x1.a01a01a01a01ap-13);
  p = dm_fma(p, r, 0x1.6c16c16c16c17p-10);
  p = dm_fma(p, r, 0x1.1111111111111p-7);
  p = dm_fma(p, r, 0x1.5555555555555p-5);
  p = dm_fma(p, r, 0x1.5555555555555p-3);
  p = dm_fma(p, r, 0x1.0000000000000p-1);
  p = dm_fma(p, r, 1.0);
  p = dm_fma(p, r, 1.0);                        /* 1/0! */
  int k1 = k / 2;
  int k2 = k - k1;
  return dm_mul(dm_mul(p, dm_pow2i(k1)), dm_pow2i(k2));
}

/* Coefficients of det_erf's two polynomials (Chebyshev interpolants in the
   scaled variable w, printed by detmath_fit.py beside this header). */
/* w = 0x1.47ae147ae147bp-2 * x^2 - 1 */
#define DBGZ_ERF_SMALL_TABLE { \
  0x1.1e08aeaa8650ap-1, -0x1.04a6751f9f826p-2, 0x1.37a6bbdd5dff1p-3, -0x1.6229127b4e09ap-4, \
  0x1.699083fd4da97p-5, -0x1.480bba23a3cf3p-6, 0x1.0932bfab89751p-7, -0x1.80a17ccd89906p-9, \
  0x1.f84117c731959p-11, -0x1.2d039dac0b9cbp-12, 0x1.49855ec9ea9a2p-14, -0x1.4ccb026cd7ac9p-16, \
  0x1.37c5543838ad3p-18, -0x1.10415382f02d3p-20, 0x1.bd28db7780427p-23, -0x1.561fd81e7b4ffp-25, \
  0x1.efc75c9366d45p-28, -0x1.518b98082c297p-30, 0x1.b78cb743bfdeep-33, -0x1.30caba530a4c6p-35, \
  0x1.642a65645191bp-38 }
/* w = 0x1.2492492492492p-1 * x - 0x1.36db6db6db6dbp+1 */
#define DBGZ_ERFC_MID_TABLE { \
  0x1.fcae93fb7323cp-30, -0x1.e55d8fd35debcp-26, 0x1.c33cfbaf8086cp-23, -0x1.0fee8de090e52p-20, \
  0x1.dcd556852b040p-19, -0x1.436a466db60bfp-17, 0x1.60392843ab955p-16, -0x1.3b48041f58d56p-15, \
  0x1.d6a728a610dd2p-15, -0x1.2711d8a329301p-14, 0x1.36cb3b28f9ca4p-14, -0x1.106827575be16p-14, \
  0x1.82eac9297cf0ap-15, -0x1.9edd47a9e41ccp-16, 0x1.008cc21c587c3p-17, 0x1.e28f4bf406f2ep-20, \
  -0x1.276826cbf28b2p-18, 0x1.b250c58e97130p-19, -0x1.53deb2980b4cep-20, 0x1.555debf6242abp-26, \
  0x1.7c75ab8562b38p-22, -0x1.246ac700ccdddp-22, 0x1.7ef1fa280d25fp-24, 0x1.9e3c953cbc15cp-26, \
  -0x1.3a07919cc4bbep-25, 0x1.484a5895a1f8ap-27, 0x1.9dc6e9fd8a5a7p-29, -0x1.db21508b6ec92p-30, \
  0x1.3c7dccdd0c1cep-33 }


DBGZ_HD double det_erf(double x) {
  if (x != x) return x;
  const double ax = fabs(x);
  double r;
  if (ax < 2.5) {
    /* erf(x) = x P(w), w = 0.32 x^2 - 1: one Horner chain of 20 fmas */
    const double c[21] = DBGZ_ERF_SMALL_TABLE;
    const double w = dm_fma(dm_mul(ax, ax), 0x1.47ae147ae147bp-2, -1.0);
    double p = c[20];
    for (int j = 19; j >= 0; --j) p = dm_fma(p, w, c[j]);
    r = dm_mul(ax, p);
  } else if (ax < 6.0) {
    /* erf(x) = 1 - Q(w), w = x / 1.75 - 17/7: one Horner chain of 28 fmas */
    const double c[29] = DBGZ_ERFC_MID_TABLE;
    const double w = dm_fma(ax, 0x1.2492492492492p-1, -0x1.36db6db6db6dbp+1);
    double q = c[28];
    for (int j = 27; j >= 0; --j) q = dm_fma(q, w, c[j]);
    r = dm_sub(1.0, q);
  } else {
    r = 1.0;  /* erfc(6) = 2.2e-17, below half an ulp of 1 */
  }
  return x < 0 ? -r : r;
}

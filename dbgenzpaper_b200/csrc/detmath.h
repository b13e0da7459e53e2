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
 * Methods (written for this library from the series definitions):
 *   exp:  x = k ln2 + r with a Cody-Waite split of ln2 (high part has 32
 *         significant bits, so k*LN2_HI is exact), degree-13 Taylor
 *         polynomial of exp(r) for |r| <= ln2/2, scaling by 2^k in two steps.
 *         Max error 1 ulp against libm on [-700, 700].
 *   erf:  |x| < 2.5: erf(x) = 2/sqrt(pi) x e^{-x^2} sum_n (2x^2)^n/(2n+1)!!
 *         (all terms positive, 51 terms, four interleaved Horner chains);
 *         2.5 <= |x| < 6:
 *         erf = 1 - erfc, erfc(x) = e^{-x^2}/(sqrt(pi) K(x)) with the
 *         Laplace continued fraction K = x + (1/2)/(x + 1/(x + (3/2)/(...)))
 *         truncated at 40 terms, evaluated by the forward recurrence of its
 *         convergents (one division);  |x| >= 6: +-1.
 *         Max error 5 ulp against libm.
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

/* 1/(2n+1)!! for n = 0..50, correctly rounded. */
#define DBGZ_DFACT_TABLE { \
  0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.1111111111111p-4, 0x1.3813813813814p-7, \
  0x1.1566abc011567p-10, 0x1.937e11175f095p-14, 0x1.f09b28ba4d955p-18, 0x1.08db48ebe51c7p-21, \
  0x1.f28db670be53bp-26, 0x1.a3d5a71b92cd3p-30, 0x1.3fdfbc45c52eap-34, 0x1.bd0ac3296b624p-39, \
  0x1.1cd3b01a822a6p-43, 0x1.519297d390c9fp-48, 0x1.747e72912d023p-53, 0x1.808286c768445p-58, \
  0x1.74dba97b8be52p-63, 0x1.54e6174c62a5ap-68, 0x1.26d4d5e132b8cp-73, 0x1.e3d36c1c38faap-79, \
  0x1.799ec4c4db4d0p-84, 0x1.19050980a3336p-89, 0x1.8fac24452c5fdp-95, 0x1.101e0dcd0ddf3p-100, \
  0x1.636b2c25f2c57p-106, 0x1.be03fb2a9a10ep-112, 0x1.0d4adb45318cap-117, 0x1.395bc2a44c468p-123, \
  0x1.5fd74f512d38cp-129, 0x1.7da878c0310ddp-135, 0x1.906d9c10fce8bp-141, 0x1.96c8bf0d31af7p-147, \
  0x1.9086a47b449d0p-153, 0x1.7e978a031f273p-159, 0x1.62de2e635bf7dp-165, 0x1.3fe183f49b037p-171, \
  0x1.18718c3c25b5ep-177, 0x1.de9fa7a781366p-184, 0x1.8dd12aeef708ap-190, 0x1.42483cb4a13e1p-196, \
  0x1.fd4910eadf32bp-203, 0x1.88b3b6aeeff5cp-209, 0x1.27ae777aaea6fp-215, 0x1.b306925c38de1p-222, \
  0x1.38d3d3acbe777p-228, 0x1.b80562010be8bp-235, 0x1.2ecf673a86d1bp-241, 0x1.97ff32292170cp-248, \
  0x1.0d319d230e257p-254, 0x1.5c0c6e1377238p-261, 0x1.b9175b58090c0p-268 }

DBGZ_HD double det_erf(double x) {
  const double TWO_OVER_SQRTPI = 0x1.20dd750429b6dp+0;
  const double INV_SQRTPI = 0x1.20dd750429b6dp-1;
  if (x != x) return x;
  double ax = fabs(x);
  double r;
  if (ax < 2.5) {
    const double c[51] = DBGZ_DFACT_TABLE;
    double x2 = dm_mul(ax, ax);
    double t = dm_add(x2, x2);
    /* s = sum_n c[n] t^n as four interleaved Horner chains in u = t^4,
       s = P0(u) + t (P1(u) + t (P2(u) + t P3(u))), P_k(u) = sum_m c[4m+k] u^m
       (a quarter of the dependent steps of one chain) */
    const double t2 = dm_mul(t, t), u = dm_mul(t2, t2);
    double p0 = c[48], p1 = c[49], p2 = c[50], p3 = c[47];
    for (int m = 11; m >= 0; --m) {
      p0 = dm_fma(p0, u, c[4 * m]);
      p1 = dm_fma(p1, u, c[4 * m + 1]);
      p2 = dm_fma(p2, u, c[4 * m + 2]);
      if (m < 11) p3 = dm_fma(p3, u, c[4 * m + 3]);
    }
    double s = dm_fma(dm_fma(dm_fma(p3, t, p2), t, p1), t, p0);
    r = dm_mul(dm_mul(dm_mul(TWO_OVER_SQRTPI, ax), det_exp(-x2)), s);
  } else if (ax < 6.0) {
    /* K = x + (1/2)/(x + (2/2)/(x + ... + (40/2)/x)), the 40-term continued
       fraction of erfc, from the forward recurrence of its convergents
       A_n = x A_{n-1} + (n/2) A_{n-2} (B_n alike) and one division: the
       two chains are independent, no division inside the loop. */
    double A2 = 1.0, A1 = ax, B2 = 0.0, B1 = 1.0;
    for (int n = 1; n <= 40; ++n) {
      const double an = dm_mul((double)n, 0.5);
      const double A = dm_fma(ax, A1, dm_mul(an, A2));
      const double B = dm_fma(ax, B1, dm_mul(an, B2));
      A2 = A1;
      A1 = A;
      B2 = B1;
      B1 = B;
    }
    const double K = dm_div(A1, B1);
    double erfc_v = dm_div(dm_mul(det_exp(-dm_mul(ax, ax)), INV_SQRTPI), K);
    r = dm_sub(1.0, erfc_v);
  } else {
    r = 1.0;
  }
  return x < 0 ? -r : r;
}

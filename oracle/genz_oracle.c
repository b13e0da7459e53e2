/*
 * genz_oracle.c -- CPU double-precision restatement of the reference's
 * qmc_pnorm! path.  TEST INFRASTRUCTURE ONLY (see genz_oracle.h).
 *
 * Each function follows the reference file:line it names.  Loops use the
 * reference's 1-based indices through the M1()/U1() accessors so that the
 * restatement can be read against the Julia line by line.  Where the
 * reference calls BLAS (mul!, ldiv!, dot) the summation order is not
 * specified by the reference; here every such sum is one fused-multiply-add
 * chain in ascending index order, the same order the GPU factorisation
 * uses, so that the pivot permutation can be compared exactly.
 *
 * Build flags must include -ffp-contract=off (explicit fma() only).
 */
#include "genz_oracle.h"
#include "../dbgenzpaper_b200/csrc/detmath.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

double orc_det_erf(double x) { return det_erf(x); }
double orc_det_exp(double x) { return det_exp(x); }

/* erfinv: Winitzki's closed-form starting value (a = 0.147), then Newton
 * steps on erf (|x| <= 0.5) or on erfc with the exactly representable
 * complement 1-|x| (|x| > 0.5). */
double orc_erfinv(double x) {
  if (x != x || x < -1.0 || x > 1.0) return NAN;
  if (x == 1.0) return INFINITY;
  if (x == -1.0) return -INFINITY;
  if (x == 0.0) return x;
  double ax = fabs(x);
  const double A = 0.147;
  const double TWO_OVER_PI_A = 2.0 / (M_PI * A);
  double w = log((1.0 - ax) * (1.0 + ax));
  double t = TWO_OVER_PI_A + 0.5 * w;
  double y = sqrt(sqrt(t * t - w / A) - t);
  const double k = 2.0 / sqrt(M_PI);
  if (ax <= 0.5) {
    for (int it = 0; it < 4; ++it) {
      double f = erf(y) - ax;
      y -= f / (k * exp(-y * y));
    }
  } else {
    double q = 1.0 - ax; /* exact for ax in [0.5, 1] */
    for (int it = 0; it < 6; ++it) {
      double f = erfc(y) - q;
      double dy = f / (k * exp(-y * y));
      y += dy;
      if (fabs(dy) <= 1e-17 * y) break;
    }
  }
  return x < 0 ? -y : y;
}

/* ------------------------------------------------------------------ */
/* Cholesky with Genz reordering: src/cholesky.jl:445-628              */
/* ------------------------------------------------------------------ */
#define M1(i, j) M[((j) - 1) * n + ((i) - 1)]
static inline int64_t imin(int64_t a, int64_t b) { return a < b ? a : b; }

/* The total order Julia's findmin/argmin uses (Base.isgreater): NaN below
 * every number, -0.0 below +0.0; ties keep the first index. */
static inline int julia_min_less(double x, double y) {
  if (x != x) return y == y;
  if (y != y) return 0;
  if (x < y) return 1;
  if (x == y && x == 0.0) return signbit(x) && !signbit(y);
  return 0;
}
static inline int64_t imax(int64_t a, int64_t b) { return a > b ? a : b; }

/* C[r,c] -= sum_l A[r,l]*B[l,c]  with the sum an ascending fma chain. */
/* ldiv!(UpperTriangular(M[p0:p1,p0:p1])', M[p0:p1, c0:c1]) */
static void trsm_upper_t(int64_t n, double *M, int64_t p0, int64_t p1, int64_t c0, int64_t c1) {
  for (int64_t c = c0; c <= c1; ++c)
    for (int64_t r = p0; r <= p1; ++r) {
      double acc = 0.0;
      for (int64_t l = p0; l < r; ++l) acc = fma(M1(l, r), M1(l, c), acc);
      M1(r, c) = (M1(r, c) - acc) / M1(r, r);
    }
}
/* mul!(M[c0:c1,c0:c1], transpose(M[p0:p1,c0:c1]), M[p0:p1,c0:c1], -1, 1) */
static void syrk_full(int64_t n, double *M, int64_t p0, int64_t p1, int64_t c0, int64_t c1) {
  for (int64_t k = c0; k <= c1; ++k)
    for (int64_t j = c0; j <= c1; ++j) {
      double acc = 0.0;
      for (int64_t l = p0; l <= p1; ++l) acc = fma(M1(l, j), M1(l, k), acc);
      M1(j, k) = M1(j, k) - acc;
    }
}

static void scale_to_correlation(int64_t n, double *M, double *a, double *b, double *scale_vec,
                                 int mirror) {
  for (int64_t j = 1; j <= n; ++j) {
    double val = M1(j, j);
    scale_vec[j - 1] = val > 0 ? sqrt(val) : 1.0;
  }
  for (int64_t j = 1; j <= n; ++j) {
    double s_j = scale_vec[j - 1];
    double inv_s_j = 1.0 / s_j;
    M1(j, j) = 1.0;
    a[j - 1] *= inv_s_j;
    b[j - 1] *= inv_s_j;
    for (int64_t i = 1; i <= j - 1; ++i) {
      double s_i = scale_vec[i - 1];
      double val = M1(i, j) * (inv_s_j / s_i);
      M1(i, j) = val;
      if (mirror) M1(j, i) = val;
    }
  }
}

static double max_abs_diag(int64_t n, const double *M) {
  double mx = 0.0;
  for (int64_t j = 1; j <= n; ++j) {
    double v = fabs(M1(j, j));
    if (v > mx || v != v) mx = v;
  }
  return mx;
}

void orc_cholesky_genz(int64_t n, double *M, double *a, double *b,
                       int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                       int64_t *perm, double *scale_vec, int64_t *rank_out) {
  orc_cholesky_genz_margins(n, M, a, b, bs1, bs2, bs3, bs4, perm, scale_vec, rank_out, NULL);
}

void orc_cholesky_genz_margins(int64_t n, double *M, double *a, double *b,
                               int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                               int64_t *perm, double *scale_vec, int64_t *rank_out, double *margins) {
  const double c2 = 1.0 / sqrt(2.0);
  const double is2pi = 2.0 / sqrt(2.0 * M_PI);
  const double eps0 = DBL_EPSILON * max_abs_diag(n, M);
  scale_to_correlation(n, M, a, b, scale_vec, 1);
  for (int64_t i = 0; i < n; ++i) perm[i] = i;
  int64_t rank = n;
  double *d_vec = (double *)calloc((size_t)n + 1, sizeof(double));
  double *s_vec = (double *)calloc((size_t)n + 1, sizeof(double));
  double *order_vec = (double *)calloc((size_t)n + 1, sizeof(double));
#define D1(k) d_vec[(k) - 1]
#define S1(k) s_vec[(k) - 1]
#define O1(k) order_vec[(k) - 1]
#define A1(k) a[(k) - 1]
#define B1(k) b[(k) - 1]
  for (int64_t iv0 = 1; iv0 <= n; iv0 += bs4) {
    int64_t iv1 = imin(n, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1; iii0 += bs3) {
      int64_t iii1 = imin(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1; ii0 += bs2) {
        int64_t ii1 = imin(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1; i0 += bs1) {
          int64_t i1 = imin(ii1, i0 + bs1 - 1);
          for (int64_t k = i0; k <= ii1; ++k) D1(k) = 0.0;
          for (int64_t i = i0; i <= i1; ++i) {
            /* pivot scores, :500-512 */
            for (int64_t k = i; k <= ii1; ++k) {
              double m_kk = M1(k, k) - D1(k);
              m_kk = m_kk < 0 ? 0.0 : sqrt(m_kk);
              double a_k = (A1(k) - S1(k)) / m_kk * c2;
              double b_k = (B1(k) - S1(k)) / m_kk * c2;
              O1(k) = det_erf(b_k) - det_erf(a_k);
            }
            /* argmin over i..ii1 (:514): first NaN wins, else first minimum */
            int64_t i_m = i;
            double best = O1(i);
            for (int64_t k = i + 1; k <= ii1; ++k) {
              double v = O1(k);
              if (julia_min_less(v, best)) { best = v; i_m = k; }
            }
            if (margins) {
              /* diagnostics, not part of the reference: the gap between the
               * winning score and the best other candidate (+inf when alone);
               * a gap near rounding size marks a pivot that a different
               * summation order could flip */
              double second = INFINITY;
              for (int64_t k = i; k <= ii1; ++k)
                if (k != i_m && O1(k) < second) second = O1(k);
              margins[i - 1] = second - best;
            }
            double d_ii = O1(i_m);
            double m_ii = M1(i_m, i_m) - D1(i_m);
            if (i_m != i) { /* :518-531 */
              int64_t tp = perm[i - 1]; perm[i - 1] = perm[i_m - 1]; perm[i_m - 1] = tp;
              double t;
              t = D1(i_m); D1(i_m) = D1(i); D1(i) = t;
              t = S1(i_m); S1(i_m) = S1(i); S1(i) = t;
              t = A1(i_m); A1(i_m) = A1(i); A1(i) = t;
              t = B1(i_m); B1(i_m) = B1(i); B1(i) = t;
              for (int64_t k = i0; k <= n; ++k) { t = M1(i, k); M1(i, k) = M1(i_m, k); M1(i_m, k) = t; }
              for (int64_t k = 1; k <= n; ++k) { t = M1(k, i); M1(k, i) = M1(k, i_m); M1(k, i_m) = t; }
            }
            if (m_ii > eps0) {
              m_ii = sqrt(m_ii);
            } else {
              rank = i - 1;
              break;
            }
            M1(i, i) = m_ii;
            double a_norm = (A1(i) - S1(i)) / m_ii;
            double b_norm = (B1(i) - S1(i)) / m_ii;
            double y_i = (det_exp(-(a_norm * a_norm) / 2.0) - det_exp(-(b_norm * b_norm) / 2.0)) * is2pi / d_ii;
            if (i == i0) { /* :547-554 */
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double m_ij = M1(i, j) / m_ii;
                M1(i, j) = m_ij;
                M1(j, i) = m_ij;
                D1(j) = D1(j) + m_ij * m_ij;
                S1(j) = S1(j) + y_i * m_ij;
              }
            } else if (i < ii1) { /* :555-570 */
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double acc = 0.0;
                for (int64_t l = i0; l <= i - 1; ++l) acc = fma(M1(j, l), M1(l, i), acc);
                M1(j, i) = M1(j, i) - acc;
              }
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double m_ij = M1(j, i);
                m_ij = m_ij / m_ii;
                M1(i, j) = m_ij;
                M1(j, i) = m_ij;
                D1(j) = D1(j) + m_ij * m_ij;
                S1(j) = S1(j) + y_i * m_ij;
              }
            }
          }
          if (rank < n) break;
          if (i1 < ii1) { /* :578-582  M[j,k] -= sum_{l=i0..i1} M[j,l] M[l,k] */
            for (int64_t k = i1 + 1; k <= ii1; ++k)
              for (int64_t j = i1 + 1; j <= ii1; ++j) {
                double acc = 0.0;
                for (int64_t l = i0; l <= i1; ++l) acc = fma(M1(j, l), M1(l, k), acc);
                M1(j, k) = M1(j, k) - acc;
              }
          }
        }
        if (rank < n) break;
        if (ii1 < iii1) { /* :589-596 */
          trsm_upper_t(n, M, ii0, ii1, ii1 + 1, iii1);
          syrk_full(n, M, ii0, ii1, ii1 + 1, iii1);
        }
      }
      if (rank < n) break;
      if (iii1 < iv1) { /* :603-610 */
        trsm_upper_t(n, M, iii0, iii1, iii1 + 1, iv1);
        syrk_full(n, M, iii0, iii1, iii1 + 1, iv1);
      }
    }
    if (rank < n) break;
    if (iv1 < n) { /* :617-624 */
      trsm_upper_t(n, M, iv0, iv1, iv1 + 1, n);
      syrk_full(n, M, iv0, iv1, iv1 + 1, n);
    }
  }
#undef D1
#undef S1
#undef O1
#undef A1
#undef B1
  free(d_vec); free(s_vec); free(order_vec);
  *rank_out = rank;
}

/* src/cholesky.jl:144-242 (no pivoting; only the upper triangle is used) */
/* ------------------------------------------------------------------ */
/* Cholesky with diagonal pivoting: src/cholesky.jl:244-432            */
/* ------------------------------------------------------------------ */
void orc_cholesky_rowmax(int64_t n, double *M, double *a, double *b,
                         int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                         int64_t *perm, double *scale_vec, int64_t *rank_out) {
  scale_to_correlation(n, M, a, b, scale_vec, 1); /* :252-271 (a, b scaled, not permuted later) */
  for (int64_t i = 0; i < n; ++i) perm[i] = i;
  int64_t rank = n;
  double *d_vec = (double *)calloc((size_t)n + 1, sizeof(double));
#define D1(k) d_vec[(k) - 1]
  for (int64_t iv0 = 1; iv0 <= n; iv0 += bs4) {
    int64_t iv1 = imin(n, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1; iii0 += bs3) {
      int64_t iii1 = imin(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1; ii0 += bs2) {
        int64_t ii1 = imin(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1; i0 += bs1) {
          int64_t i1 = imin(ii1, i0 + bs1 - 1);
          for (int64_t k = i0; k <= ii1; ++k) D1(k) = 0.0;
          for (int64_t i = i0; i <= i1; ++i) {
            /* largest remaining diagonal of the panel, first on ties (:294-305) */
            int64_t i_m = i;
            double m_ii = M1(i, i) - D1(i);
            for (int64_t k = i; k <= ii1; ++k) {
              double m_kk = M1(k, k) - D1(k);
              if (m_kk > m_ii) { m_ii = m_kk; i_m = k; }
            }
            if (m_ii > 0) { /* :309-314: the rank test comes before the swap */
              m_ii = sqrt(m_ii);
            } else {
              rank = i - 1;
              break;
            }
            if (i_m != i) { /* :316-326 (a and b are not swapped) */
              int64_t tp = perm[i - 1]; perm[i - 1] = perm[i_m - 1]; perm[i_m - 1] = tp;
              double t = D1(i_m); D1(i_m) = D1(i); D1(i) = t;
              for (int64_t k = i0; k <= n; ++k) { t = M1(i, k); M1(i, k) = M1(i_m, k); M1(i_m, k) = t; }
              for (int64_t k = 1; k <= n; ++k) { t = M1(k, i); M1(k, i) = M1(k, i_m); M1(k, i_m) = t; }
            }
            M1(i, i) = m_ii;
            if (i == i0) { /* :332-338 */
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double m_ij = M1(i, j) / m_ii;
                M1(i, j) = m_ij;
                M1(j, i) = m_ij;
                D1(j) = D1(j) + m_ij * m_ij;
              }
            } else if (i < ii1) { /* :339-353 */
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double acc = 0.0;
                for (int64_t l = i0; l <= i - 1; ++l) acc = fma(M1(j, l), M1(l, i), acc);
                M1(j, i) = M1(j, i) - acc;
              }
              for (int64_t j = i + 1; j <= ii1; ++j) {
                double m_ij = M1(j, i);
                m_ij = m_ij / m_ii;
                M1(i, j) = m_ij;
                M1(j, i) = m_ij;
                D1(j) = D1(j) + m_ij * m_ij;
              }
            }
          }
          if (rank < n) break;
          if (i1 < ii1) { /* :361-365 */
            for (int64_t k = i1 + 1; k <= ii1; ++k)
              for (int64_t j = i1 + 1; j <= ii1; ++j) {
                double acc = 0.0;
                for (int64_t l = i0; l <= i1; ++l) acc = fma(M1(j, l), M1(l, k), acc);
                M1(j, k) = M1(j, k) - acc;
              }
          }
        }
        if (rank < n) break;
        if (ii1 < iii1) { /* :372-379 */
          trsm_upper_t(n, M, ii0, ii1, ii1 + 1, iii1);
          syrk_full(n, M, ii0, ii1, ii1 + 1, iii1);
        }
      }
      if (rank < n) break;
      if (iii1 < iv1) { /* :385-392 */
        trsm_upper_t(n, M, iii0, iii1, iii1 + 1, iv1);
        syrk_full(n, M, iii0, iii1, iii1 + 1, iv1);
      }
    }
    if (rank < n) break;
    if (iv1 < n) { /* :398-405 */
      trsm_upper_t(n, M, iv0, iv1, iv1 + 1, n);
      syrk_full(n, M, iv0, iv1, iv1 + 1, n);
    }
  }
#undef D1
  free(d_vec);
  *rank_out = rank;
}

/* ------------------------------------------------------------------ */
/* adapt_low_rank!: src/cholesky.jl:24-123                             */
/* ------------------------------------------------------------------ */
void orc_adapt_low_rank(int64_t nr, int64_t n, double *M, double *a, double *b, int64_t rank, int64_t *perm,
                        double eps1, int64_t *k_js, int64_t *k_0_out) {
  /* M is nr x n (column-major); k_js (length rank) receives the 1-based
   * block ends; perm holds 0-based indices and is permuted in place */
#define MC(i, j) M[((j) - 1) * nr + ((i) - 1)]
  double *tmp = (double *)malloc(sizeof(double) * (size_t)(nr > 0 ? nr : 1));
  for (int64_t i = 1; i <= rank; ++i) k_js[i - 1] = i;
  int64_t k_0 = 0, j = rank + 1, n_active = n;
  while (j <= n_active) {
    /* level: last row i <= rank with |M[i, j]| > eps1 (:41) */
    int64_t i_j = 0;
    for (int64_t i = rank; i >= 1; --i)
      if (fabs(MC(i, j)) > eps1) { i_j = i; break; }
    if (i_j == 0) { /* :44-61: to the end, not advancing j */
      if (j != n_active) {
        for (int64_t r = 1; r <= nr; ++r) { double t = MC(r, n_active); MC(r, n_active) = MC(r, j); MC(r, j) = t; }
        double t = a[j - 1]; a[j - 1] = a[n_active - 1]; a[n_active - 1] = t;
        t = b[j - 1]; b[j - 1] = b[n_active - 1]; b[n_active - 1] = t;
        int64_t tp = perm[j - 1]; perm[j - 1] = perm[n_active - 1]; perm[n_active - 1] = tp;
      }
      k_0 += 1;
      n_active -= 1;
      continue;
    }
    /* :64-80: scale by the pivot, swap the bounds if it is negative */
    double m_ij = MC(i_j, j);
    int is_neg = m_ij < 0.0;
    double inv_m = 1.0 / m_ij;
    for (int64_t k = 1; k <= i_j; ++k) MC(k, j) *= inv_m;
    a[j - 1] *= inv_m;
    b[j - 1] *= inv_m;
    if (is_neg) { double t = a[j - 1]; a[j - 1] = b[j - 1]; b[j - 1] = t; }
    /* :85-111: insert at the end of block i_j */
    int64_t pos = k_js[i_j - 1] + 1;
    if (j != pos) {
      for (int64_t r = 1; r <= nr; ++r) tmp[r - 1] = MC(r, j);
      double va = a[j - 1], vb = b[j - 1];
      int64_t vp = perm[j - 1];
      for (int64_t c = j; c >= pos + 1; --c) {
        for (int64_t r = 1; r <= nr; ++r) MC(r, c) = MC(r, c - 1);
        a[c - 1] = a[c - 2];
        b[c - 1] = b[c - 2];
        perm[c - 1] = perm[c - 2];
      }
      for (int64_t r = 1; r <= nr; ++r) MC(r, pos) = tmp[r - 1];
      a[pos - 1] = va;
      b[pos - 1] = vb;
      perm[pos - 1] = vp;
    }
    for (int64_t k = i_j; k <= rank; ++k) k_js[k - 1] += 1; /* :115-118 */
    j += 1;
  }
#undef MC
  free(tmp);
  *k_0_out = k_0;
}

void orc_cholesky_classic(int64_t n, double *M, double *a, double *b,
                          int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                          double *scale_vec) {
  scale_to_correlation(n, M, a, b, scale_vec, 0);
  for (int64_t iv0 = 1; iv0 <= n; iv0 += bs4) {
    int64_t iv1 = imin(n, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1; iii0 += bs3) {
      int64_t iii1 = imin(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1; ii0 += bs2) {
        int64_t ii1 = imin(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1; i0 += bs1) {
          int64_t i1 = imin(ii1, i0 + bs1 - 1);
          for (int64_t i = i0; i <= i1; ++i) {
            double m_ii = M1(i, i);
            if (i > i0) {
              double acc = 0.0;
              for (int64_t l = i0; l <= i - 1; ++l) acc = fma(M1(l, i), M1(l, i), acc);
              m_ii -= acc;
            }
            m_ii = sqrt(m_ii);
            M1(i, i) = m_ii;
            if (i > i0 && i < i1) {
              for (int64_t j = i + 1; j <= i1; ++j) {
                double acc = 0.0;
                for (int64_t l = i0; l <= i - 1; ++l) acc = fma(M1(l, j), M1(l, i), acc);
                M1(i, j) -= acc;
                M1(j, i) = 0.0;
              }
            }
            for (int64_t j = i + 1; j <= i1; ++j) M1(i, j) /= m_ii;
          }
          if (i1 < ii1) {
            trsm_upper_t(n, M, i0, i1, i1 + 1, ii1);
            syrk_full(n, M, i0, i1, i1 + 1, ii1);
          }
        }
        if (ii1 < iii1) {
          trsm_upper_t(n, M, ii0, ii1, ii1 + 1, iii1);
          syrk_full(n, M, ii0, ii1, ii1 + 1, iii1);
        }
      }
      if (iii1 < iv1) {
        trsm_upper_t(n, M, iii0, iii1, iii1 + 1, iv1);
        syrk_full(n, M, iii0, iii1, iii1 + 1, iv1);
      }
    }
    if (iv1 < n) {
      trsm_upper_t(n, M, iv0, iv1, iv1 + 1, n);
      syrk_full(n, M, iv0, iv1, iv1 + 1, n);
    }
  }
}
#undef M1

/* src/qmc.jl:133-142 */
void orc_truncate_U(int64_t n, double *U, double eps_T) {
  double min_val = eps_T / (double)(n * 9);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < n; ++i)
      if (fabs(U[j * n + i]) < min_val) U[j * n + i] = 0.0;
}

/* ------------------------------------------------------------------ */
/* Point generators: src/qmc_generators.jl:300-325, Sobol (Gray code)  */
/* ------------------------------------------------------------------ */
static int is_prime(int64_t p) {
  if (p < 2) return 0;
  for (int64_t f = 2; f * f <= p; ++f) if (p % f == 0) return 0;
  return 1;
}
void orc_sqrt_primes(int64_t n, double *q) {
  int64_t p = 1;
  for (int64_t i = 0; i < n; ++i) {
    p = p + 1;
    while (!is_prime(p)) ++p; /* nextprime(p + 1) */
    double sp = sqrt((double)p);
    q[i] = sp - floor(sp);
  }
}
void orc_richtmyer_mat(int64_t m, int64_t n, const double *q, int64_t n0, double *X) {
  for (int64_t j = 0; j < n; ++j) {
    double qj = q[j];
    for (int64_t i = 1; i <= m; ++i) {
      double x = (double)(n0 + i) * qj;
      X[j * m + (i - 1)] = x - floor(x);
    }
  }
}
void orc_sobol_points(int64_t dims, const uint32_t *V, int64_t first, int64_t m, uint32_t *X) {
  for (int64_t j = 0; j < m; ++j) {
    uint64_t idx = (uint64_t)(first + j);
    uint64_t g = idx ^ (idx >> 1);
    for (int64_t i = 0; i < dims; ++i) {
      uint32_t x = 0;
      for (int k = 0; k < 32; ++k)
        if ((g >> k) & 1u) x ^= V[i * 32 + k];
      X[i * m + j] = x;
    }
  }
}

/* ------------------------------------------------------------------ */
/* Integration loop: src/qmc.jl:315-444 / :485-608 / :618-718          */
/* ------------------------------------------------------------------ */
typedef struct tile_buf {
  double *Y, *S, *c, *dc, *p;
  double *lw; /* per-sample sum of log dc (the log of p), when P->logw is set */
} tile_buf;

static inline double clamp9(double v) { return fmax(fmin(v, 9.0), -9.0); }

/* rand_points!: src/qmc_generators.jl:137-165 (Richtmyer) and :175-204 (Sobol).
 * Fills column i (1-based) of Y for the tile rows. */
static void rand_points(const orc_problem *P, const orc_opts *o, int64_t n_pass_base,
                        int64_t j1, int64_t len, int64_t i, int64_t k, tile_buf *tb) {
  const int64_t n = P->n;
  const double ep0 = DBL_EPSILON, ep1 = 1.0 - DBL_EPSILON;
  double *Yc = tb->Y + (i - 1) * len;
  if (P->qmc_type == ORC_RICHTMYER) {
    double shift = P->shifts[(k - 1) * (n - 1) + (i - 1)];
    double qi = P->q[i - 1];
    for (int64_t t = 0; t < len; ++t) {
      int64_t j = j1 + t; /* 1-based point index within the pass */
      double x = (double)(n_pass_base + j) * qi;
      x = x - floor(x);
      double u = shift + x;
      u = u > 1.0 ? u - 1.0 : u;
      u = fabs(fma(u, 2.0, -1.0));
      u = fma(u, tb->dc[t], tb->c[t]);
      u = fmin(fmax(u, ep0), ep1);
      Yc[t] = fma(2.0, u, -1.0);
    }
  } else {
    const int L = (int)o->n_bits;
    const uint64_t mask = (L >= 64) ? ~(uint64_t)0 : (((uint64_t)1 << L) - 1);
    const double invscale = ldexp(1.0, -L);
    uint64_t shift = P->ushifts[(k - 1) * (n - 1) + (i - 1)] & mask;
    const uint32_t *Vi = P->V + (i - 1) * 32;
    for (int64_t t = 0; t < len; ++t) {
      uint64_t idx = (uint64_t)(P->sobol_first + n_pass_base + j1 + t - 1);
      uint64_t g = idx ^ (idx >> 1);
      uint32_t xi = 0;
      for (int b = 0; b < 32; ++b) if ((g >> b) & 1u) xi ^= Vi[b];
      uint64_t x_ij = (uint64_t)xi & mask;
      double u = (double)((x_ij ^ shift) & mask) * invscale;
      u = fabs(fma(u, 2.0, -1.0));
      u = fma(u, tb->dc[t], tb->c[t]);
      u = fmin(fmax(u, ep0), ep1);
      Yc[t] = fma(2.0, u, -1.0);
    }
  }
}

static void cdf_update(const orc_problem *P, double a_i, double b_i, double inv_u, const double *scol,
                       int64_t len, tile_buf *tb) {
  for (int64_t t = 0; t < len; ++t) {
    double s = scol[t];
    double cv = (a_i - s) * inv_u;
    double dv = (b_i - s) * inv_u;
    if (P->cdf_form == ORC_CDF_ERF) {
      cv = erf(clamp9(cv));
      dv = erf(clamp9(dv));
      cv = 0.5 * (1.0 + cv);
      dv = 0.5 * (1.0 + dv) - cv;
    } else {
      cv = clamp9(cv);
      dv = clamp9(dv);
      double c_val = 0.5 * erfc(-cv);
      dv = 0.5 * erfc(-dv) - c_val;
      cv = c_val;
    }
    tb->c[t] = cv;
    tb->dc[t] = dv;
    tb->p[t] *= dv;
    if (tb->lw) tb->lw[t] += log(dv);
  }
}

static double dense_tile(const orc_problem *P, const orc_opts *o, int64_t bi, int64_t bi2,
                         int64_t n_pass_base, int64_t j1, int64_t len, int64_t k,
                         double c_1, double dc_1, tile_buf *tb) {
  const int64_t n = P->n;
  const double *U = P->U;
  const double c2 = sqrt(2.0);
#define U1(i, j) U[((j) - 1) * n + ((i) - 1)]
#define Y1(t, i) tb->Y[((i) - 1) * len + (t)]
#define S1(t, c) tb->S[((c) - 1) * len + (t)]
  for (int64_t t = 0; t < len; ++t) { tb->c[t] = c_1; tb->dc[t] = dc_1; tb->p[t] = dc_1; }
  if (tb->lw) for (int64_t t = 0; t < len; ++t) tb->lw[t] = log(dc_1);
  memset(tb->S, 0, sizeof(double) * (size_t)(len * bi));
  for (int64_t ii1 = 1; ii1 <= n - 1; ii1 += bi) {
    int64_t ii2 = imin(ii1 + bi - 1, n - 1);
    if (ii1 > 1) { /* :350-362 */
      for (int64_t col = 1; col <= ii2 - ii1 + 1; ++col) {
        int64_t tgt = ii1 + col;
        for (int64_t t = 0; t < len; ++t) {
          double acc = 0.0;
          for (int64_t l = 1; l <= ii1 - 1; ++l) acc = fma(Y1(t, l), U1(l, tgt), acc);
          S1(t, col) = acc;
        }
      }
    }
    for (int64_t i1 = ii1; i1 <= ii2; i1 += bi2) {
      int64_t i2 = imin(i1 + bi2 - 1, ii2);
      if (i1 > ii1) { /* :367-378 */
        int64_t prev1 = imax(ii1, i1 - bi2), prev2 = i1 - 1;
        for (int64_t col = i1 - ii1 + 1; col <= ii2 - ii1 + 1; ++col) {
          int64_t tgt = ii1 + col;
          for (int64_t t = 0; t < len; ++t) {
            double acc = 0.0;
            for (int64_t l = prev1; l <= prev2; ++l) acc = fma(Y1(t, l), U1(l, tgt), acc);
            S1(t, col) = S1(t, col) + acc;
          }
        }
      }
      for (int64_t i = i1; i <= i2; ++i) {
        rand_points(P, o, n_pass_base, j1, len, i, k, tb);
        for (int64_t t = 0; t < len; ++t) Y1(t, i) = c2 * orc_erfinv(Y1(t, i));
        int64_t scol = i - ii1 + 1;
        for (int64_t t = 0; t < len; ++t) { /* :394-403 */
          double acc = S1(t, scol);
          for (int64_t kk = i1; kk <= i; ++kk) acc = fma(Y1(t, kk), U1(kk, i + 1), acc);
          S1(t, scol) = acc;
        }
        double inv_u = 1.0 / (U1(i + 1, i + 1) * c2);
        cdf_update(P, P->a[i], P->b[i], inv_u, &S1(0, scol), len, tb);
      }
    }
  }
  double sum = 0.0;
  for (int64_t t = 0; t < len; ++t) sum += tb->p[t];
  return sum;
#undef U1
#undef Y1
#undef S1
}

/* sparse loop :618-718 over the strict upper CSC of U (ascending rows) */
typedef struct csc { int64_t *colptr; int64_t *rowval; double *nzval; } csc;

static double sparse_tile(const orc_problem *P, const orc_opts *o, const csc *C,
                          int64_t n_pass_base, int64_t j1, int64_t len, int64_t k,
                          double c_1, double dc_1, tile_buf *tb) {
  const int64_t n = P->n;
  const double c2 = sqrt(2.0);
  for (int64_t t = 0; t < len; ++t) { tb->c[t] = c_1; tb->dc[t] = dc_1; tb->p[t] = dc_1; }
  if (tb->lw) for (int64_t t = 0; t < len; ++t) tb->lw[t] = log(dc_1);
  for (int64_t i = 1; i <= n - 1; ++i) {
    rand_points(P, o, n_pass_base, j1, len, i, k, tb);
    double *Yi = tb->Y + (i - 1) * len;
    for (int64_t t = 0; t < len; ++t) Yi[t] = c2 * orc_erfinv(Yi[t]);
    for (int64_t t = 0; t < len; ++t) tb->S[t] = 0.0;
    /* column i+1 (1-based) is index i (0-based) */
    for (int64_t pp = C->colptr[i]; pp < C->colptr[i + 1]; ++pp) {
      int64_t iu = C->rowval[pp]; /* 0-based row */
      double v = C->nzval[pp];
      const double *Yr = tb->Y + iu * len;
      for (int64_t t = 0; t < len; ++t) tb->S[t] = fma(Yr[t], v, tb->S[t]);
    }
    double inv_u = 1.0 / (P->U[i * n + i] * c2);
    orc_problem Pe = *P; Pe.cdf_form = ORC_CDF_ERF; /* the sparse loop has only the erf form */
    cdf_update(&Pe, P->a[i], P->b[i], inv_u, tb->S, len, tb);
  }
  double sum = 0.0;
  for (int64_t t = 0; t < len; ++t) sum += tb->p[t];
  return sum;
}

/* sd(): src/qmc.jl:303-312 */
static double sd_ref(const double *v, int64_t n, double mean) {
  double r = 0.0;
  for (int64_t i = 0; i < n; ++i) { double d = v[i] - mean; r += d * d / (double)n; }
  return sqrt(r / (double)(n - 1));
}

static void qmc_loop(const orc_problem *P, const orc_opts *o, const csc *C, int threads,
                     int64_t n_pts0, int64_t n_pass_base, double c_1, double dc_1, double *reps) {
  const int64_t n = P->n;
  int64_t bi = o->block_size_i, bi2 = o->block_size_i2;
  if (n - 1 < o->block_size_i) { /* QMCData clamp, src/qmc.jl:166-174 */
    bi = n - 1;
    if (n - 1 < o->block_size_i2) bi2 = n - 1;
  }
  const int64_t bj = o->block_size_j, m = o->m;
  const int64_t n_tiles = (m + bj - 1) / bj;
  double *tile_sums = (double *)malloc(sizeof(double) * (size_t)n_tiles);
  for (int64_t k = 1; k <= o->n_reps; ++k) {
#pragma omp parallel num_threads(threads > 0 ? threads : omp_get_max_threads())
    {
      tile_buf tb;
      tb.Y = (double *)malloc(sizeof(double) * (size_t)(bj * (n > 1 ? n - 1 : 1)));
      tb.S = (double *)malloc(sizeof(double) * (size_t)(bj * (bi > 1 ? bi : 1)));
      tb.c = (double *)malloc(sizeof(double) * (size_t)bj);
      tb.dc = (double *)malloc(sizeof(double) * (size_t)bj);
      tb.p = (double *)malloc(sizeof(double) * (size_t)bj);
      tb.lw = P->logw ? (double *)malloc(sizeof(double) * (size_t)bj) : NULL;
#pragma omp for schedule(dynamic, 1)
      for (int64_t tt = 0; tt < n_tiles; ++tt) {
        int64_t j1 = 1 + tt * bj;
        int64_t j2 = imin(j1 + bj - 1, m);
        int64_t len = j2 - j1 + 1;
        tile_sums[tt] = P->sparse
            ? sparse_tile(P, o, C, n_pass_base, j1, len, k, c_1, dc_1, &tb)
            : dense_tile(P, o, bi, bi2, n_pass_base, j1, len, k, c_1, dc_1, &tb);
        if (P->logw) memcpy(P->logw + (k - 1) * m + (j1 - 1), tb.lw, sizeof(double) * (size_t)len);
      }
      free(tb.Y); free(tb.S); free(tb.c); free(tb.dc); free(tb.p); free(tb.lw);
    }
    double total = 0.0;
    for (int64_t tt = 0; tt < n_tiles; ++tt) total += tile_sums[tt];
    int64_t n_pts_total = n_pts0 + m;
    double inv_tot = 1.0 / (double)n_pts_total;
    double mean_rep = total * inv_tot;
    double old_weight = (double)n_pts0 * inv_tot;
    reps[k - 1] = fma(reps[k - 1], old_weight, mean_rep);
  }
  free(tile_sums);
}

void orc_qmc_pnorm(const orc_problem *P, const orc_opts *o, int threads,
                   double *result, double *err, int64_t *n_pts_out, double *reps) {
  const int64_t n = P->n;
  const int64_t n_reps = o->n_reps;
  csc C = {0, 0, 0};
  if (P->sparse) { /* U_S = sparse(triu(U, 1)), src/qmc.jl:272-279 */
    C.colptr = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t nnz = 0;
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i = 0; i < j; ++i) if (P->U[j * n + i] != 0.0) ++nnz;
    C.rowval = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nnz + 1));
    C.nzval = (double *)malloc(sizeof(double) * (size_t)(nnz + 1));
    int64_t pp = 0;
    for (int64_t j = 0; j < n; ++j) {
      C.colptr[j] = pp;
      for (int64_t i = 0; i < j; ++i)
        if (P->U[j * n + i] != 0.0) { C.rowval[pp] = i; C.nzval[pp] = P->U[j * n + i]; ++pp; }
    }
    C.colptr[n] = pp;
  }
  for (int64_t k = 0; k < n_reps; ++k) reps[k] = 0.0;
  const double sq2 = sqrt(2.0);
  double arg_a = P->a[0] / (P->U[0] * sq2);
  double arg_b = P->b[0] / (P->U[0] * sq2);
  double c_1, dc_1;
  if (P->cdf_form == ORC_CDF_ERFC && !P->sparse) {
    c_1 = 0.5 * erfc(-arg_a);
    dc_1 = 0.5 * (erfc(-arg_b) - erfc(-arg_a));
  } else {
    c_1 = 0.5 * (1.0 + erf(arg_a));
    dc_1 = 0.5 * (erf(arg_b) - erf(arg_a));
  }
  int64_t n_pts = 0, n_pass_base = P->gen_base0;
  qmc_loop(P, o, &C, threads, n_pts, n_pass_base, c_1, dc_1, reps);
  double res = 0.0;
  for (int64_t k = 0; k < n_reps; ++k) res += reps[k];
  res /= (double)n_reps;
  double e = 3.0 * sd_ref(reps, n_reps, res);
  n_pts += o->m;
  while (!(n_pts >= o->max_pts || e < o->max_abs_err) && (n_pts < o->max_pts && e > o->max_abs_err)) {
    n_pass_base += o->m; /* next_points!, src/qmc_generators.jl:119-131 */
    qmc_loop(P, o, &C, threads, n_pts, n_pass_base, c_1, dc_1, reps);
    res = 0.0;
    for (int64_t k = 0; k < n_reps; ++k) res += reps[k];
    res /= (double)n_reps;
    e = 3.0 * sd_ref(reps, n_reps, res);
    n_pts += o->m;
  }
  if (P->sparse) { free(C.colptr); free(C.rowval); free(C.nzval); }
  *result = res;
  *err = e;
  *n_pts_out = n_pts;
}

/*
 * genz_cpu_blas.c -- the reference's Float64 qmc_loop! as it runs on a CPU:
 * the timed CPU baseline of bench.py (its cpu_baseline leg and the
 * --impl reference arm).  CPU-BASELINE INFRASTRUCTURE ONLY, like the checker in
 * genz_oracle.c: nothing in dbgenzpaper_b200/ links or calls it.
 *
 * Where genz_oracle.c restates the reference for exact comparison (scalar
 * fused-multiply-add chains in a fixed order, a Newton-iterated erfinv), this
 * file restates it for speed, the way the reference itself runs
 * (src/qmc.jl:315-444):
 *   - point tiles of block_size_j points spread over threads (the @batch
 *     loop, src/qmc.jl:332; OpenMP here), shifts one after another (:328);
 *   - the off-block contraction as BLAS-3 dgemm (mul!, :350-362 and :367-378)
 *     from the OpenBLAS that numpy ships, one BLAS thread per worker (the
 *     reference sets BLAS.set_num_threads(1) inside the loop, :793-796);
 *   - rand_points! (src/qmc_generators.jl:137-204), the in-block dot
 *     (:394-403) and the CDFs (:405-429) as vectorised loops over the tile,
 *     erf from glibc's vector math library (libmvec; the reference's @turbo
 *     erf is SLEEF vector code, max error 2 ulp);
 *   - erfinv (:385-387) vectorised too: a start value from a polynomial in
 *     M. Giles' form (erfinv(x) = x P(w - 2.5) for w = -ln(1 - x^2) < 5, a
 *     polynomial in sqrt(w) above; coefficients fitted for this library)
 *     refined by one Halley step on erfc(x) = 1 - |x| with libmvec's erfc and
 *     exp (the start is within 1e-7, one Halley step leaves ~1e-20 relative,
 *     so the result is as accurate as erfc itself).
 * Results agree with the checker to ~1e-13 relative (different erf, erfinv
 * and summation order); tests/test_oracle.py checks that.
 *
 * Built twice by the Makefile (AVX2 and AVX-512); the Python side loads the
 * one the CPU supports.
 */
#include <dlfcn.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

/* vector variants from glibc's libmvec (x86_64: AVX2 and AVX-512 forms) */
#pragma omp declare simd notinbranch
double erf(double);
#pragma omp declare simd notinbranch
double erfc(double);
#pragma omp declare simd notinbranch
double exp(double);
#pragma omp declare simd notinbranch
double log(double);

/* ---- BLAS (ILP64 CBLAS of numpy's OpenBLAS, bound at run time) ---------- */
typedef void (*dgemm_fn)(int, int, int, int64_t, int64_t, int64_t, double, const double *, int64_t,
                         const double *, int64_t, double, double *, int64_t);
typedef void (*set_threads_fn)(int);
typedef int (*get_threads_fn)(void);
static dgemm_fn g_dgemm;
static set_threads_fn g_set_threads;
static get_threads_fn g_get_threads;
enum { kColMajor = 102, kNoTrans = 111 };

/* Binds dgemm from the OpenBLAS shared library at `path` (numpy's bundled
 * libscipy_openblas64_: symbols scipy_cblas_dgemm64_ and friends).
 * Returns 0 on success. */
int cpu_blas_init(const char *path) {
  void *h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
  if (!h) return 1;
  g_dgemm = (dgemm_fn)dlsym(h, "scipy_cblas_dgemm64_");
  g_set_threads = (set_threads_fn)dlsym(h, "scipy_openblas_set_num_threads64_");
  g_get_threads = (get_threads_fn)dlsym(h, "scipy_openblas_get_num_threads64_");
  return (g_dgemm && g_set_threads && g_get_threads) ? 0 : 2;
}

/* ---- small GEMM for the loop's shapes (AVX-512 build) ----------------------
 * C[M x N] (+)= A[M x K] B[K x N], all column-major, M a multiple of 8 up to
 * the tile height (block_size_j), K up to block_size_i: the reference's mul!
 * calls of one tile.  Register blocking of 32 rows x 6 columns (24 zmm
 * accumulators), A streamed from L1/L2 (the tile's Y block), each B entry
 * broadcast once per 32 rows.  Stands in for the small-matrix paths of the
 * BLAS the reference's published Intel runs used (MKL); OpenBLAS repacks
 * both operands on every call at these sizes.  beta is 0 or 1. */
#if defined(__AVX512F__)
#include <immintrin.h>
#define HAVE_OWN_GEMM 1
/* 32 x NC block, NC <= 6 fixed at compile time so the accumulators stay in
 * registers */
#define GEMM_BLOCK(NAME, MR, NC)                                                                          \
  static void NAME(int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb, double beta,  \
                   double *Cm, int64_t ldc) {                                                             \
    __m512d acc[NC][MR / 8];                                                                              \
    for (int j = 0; j < NC; ++j)                                                                          \
      for (int r = 0; r < MR / 8; ++r) acc[j][r] = _mm512_setzero_pd();                                   \
    for (int64_t k = 0; k < K; ++k) {                                                                     \
      const double *a = A + k * lda;                                                                      \
      __m512d av[MR / 8];                                                                                 \
      for (int r = 0; r < MR / 8; ++r) av[r] = _mm512_loadu_pd(a + 8 * r);                                \
      for (int j = 0; j < NC; ++j) {                                                                      \
        const __m512d bj = _mm512_set1_pd(B[j * ldb + k]);                                                \
        for (int r = 0; r < MR / 8; ++r) acc[j][r] = _mm512_fmadd_pd(av[r], bj, acc[j][r]);               \
      }                                                                                                   \
    }                                                                                                     \
    for (int j = 0; j < NC; ++j)                                                                          \
      for (int r = 0; r < MR / 8; ++r) {                                                                  \
        double *c = Cm + j * ldc + 8 * r;                                                                 \
        _mm512_storeu_pd(c, beta != 0.0 ? _mm512_add_pd(_mm512_loadu_pd(c), acc[j][r]) : acc[j][r]);     \
      }                                                                                                   \
  }
GEMM_BLOCK(gemm_32x6, 32, 6)
GEMM_BLOCK(gemm_32x1, 32, 1)
GEMM_BLOCK(gemm_8x6, 8, 6)
GEMM_BLOCK(gemm_8x1, 8, 1)
static void own_dgemm(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
                      double beta, double *Cm, int64_t ldc) {
  int64_t j0 = 0;
  for (; j0 + 6 <= N; j0 += 6) {
    int64_t r0 = 0;
    for (; r0 + 32 <= M; r0 += 32) gemm_32x6(K, A + r0, lda, B + j0 * ldb, ldb, beta, Cm + j0 * ldc + r0, ldc);
    for (; r0 < M; r0 += 8) gemm_8x6(K, A + r0, lda, B + j0 * ldb, ldb, beta, Cm + j0 * ldc + r0, ldc);
  }
  for (; j0 < N; ++j0) {
    int64_t r0 = 0;
    for (; r0 + 32 <= M; r0 += 32) gemm_32x1(K, A + r0, lda, B + j0 * ldb, ldb, beta, Cm + j0 * ldc + r0, ldc);
    for (; r0 < M; r0 += 8) gemm_8x1(K, A + r0, lda, B + j0 * ldb, ldb, beta, Cm + j0 * ldc + r0, ldc);
  }
}
#endif

/* ---- erfinv ------------------------------------------------------------- */
#pragma omp declare simd notinbranch
static inline double erfinv_v(double v) {
  const double a = fabs(v);
  const double w1 = 1.0 - a; /* exact for a >= 1/2 */
  /* start value: erfinv(a) with w = -ln(1 - a^2) (Giles' variable) */
  const double w = -log(w1 * (1.0 + a));
  const double tc = w - 2.5;
  double pc = 2.854775242e-08;
  pc = fma(pc, tc, 3.437494356e-07);
  pc = fma(pc, tc, -3.528993161e-06);
  pc = fma(pc, tc, -4.396994196e-06);
  pc = fma(pc, tc, 2.186026004e-04);
  pc = fma(pc, tc, -1.253706953e-03);
  pc = fma(pc, tc, -4.177708101e-03);
  pc = fma(pc, tc, 2.466407258e-01);
  pc = fma(pc, tc, 1.501409422e+00);
  const double ts = sqrt(w) - 4.0;
  double pt = 8.193106379e-07;
  pt = fma(pt, ts, -1.490730122e-06);
  pt = fma(pt, ts, -6.624017282e-06);
  pt = fma(pt, ts, 2.765589313e-05);
  pt = fma(pt, ts, -8.117484620e-05);
  pt = fma(pt, ts, 2.877970689e-04);
  pt = fma(pt, ts, -8.563289957e-04);
  pt = fma(pt, ts, 1.256645993e-03);
  pt = fma(pt, ts, 1.009495442e+00);
  pt = fma(pt, ts, 3.839783388e+00);
  double x = w < 5.0 ? pc * a : pt;
  /* one Halley step on f(x) = erfc(x) - (1 - a):
   *   f' = -2/sqrt(pi) exp(-x^2),  f''/(2 f') = -x,
   *   x <- x - d / (1 + x d),  d = f / f' */
  const double fp = -1.1283791670955126 * exp(-x * x);
  const double f = erfc(x) - w1;
  const double dd = f / fp;
  x = x - dd / fma(x, dd, 1.0);
  return v < 0.0 ? -x : x;
}

static void gemm(int64_t M, int64_t N, int64_t K, const double *A, int64_t lda, const double *B, int64_t ldb,
                 double beta, double *Cm, int64_t ldc) {
  if (M <= 0 || N <= 0) return;
  if (K <= 0) {
    if (beta == 0.0)
      for (int64_t j = 0; j < N; ++j) memset(Cm + j * ldc, 0, sizeof(double) * (size_t)M);
    return;
  }
#ifdef HAVE_OWN_GEMM
  own_dgemm(M, N, K, A, lda, B, ldb, beta, Cm, ldc);
#else
  g_dgemm(kColMajor, kNoTrans, kNoTrans, M, N, K, 1.0, A, lda, B, ldb, beta, Cm, ldc);
#endif
}

/* sc[t] += sum_kk Y[t, kk] u[kk] for t < M (M a multiple of 8), kk < nk, the
 * sum over kk in ascending order per row (src/qmc.jl:394-403) */
static void inblock_dot(int64_t M, int nk, const double *Yb, int64_t ld, const double *u, double *sc) {
#ifdef HAVE_OWN_GEMM
  /* rows in registers, 8 vectors (64 rows) at a time */
  for (int64_t r0 = 0; r0 < M; r0 += 64) {
    const int nv = (int)((M - r0) / 8 < 8 ? (M - r0) / 8 : 8);
    __m512d acc[8];
    for (int v = 0; v < 8; ++v) acc[v] = v < nv ? _mm512_loadu_pd(sc + r0 + 8 * v) : _mm512_setzero_pd();
    if (nv == 8) {
      for (int kk = 0; kk < nk; ++kk) {
        const __m512d uk = _mm512_set1_pd(u[kk]);
        const double *y = Yb + kk * ld + r0;
        for (int v = 0; v < 8; ++v) acc[v] = _mm512_fmadd_pd(_mm512_loadu_pd(y + 8 * v), uk, acc[v]);
      }
    } else {
      for (int kk = 0; kk < nk; ++kk) {
        const __m512d uk = _mm512_set1_pd(u[kk]);
        const double *y = Yb + kk * ld + r0;
        for (int v = 0; v < nv; ++v) acc[v] = _mm512_fmadd_pd(_mm512_loadu_pd(y + 8 * v), uk, acc[v]);
      }
    }
    for (int v = 0; v < nv; ++v) _mm512_storeu_pd(sc + r0 + 8 * v, acc[v]);
  }
#else
  for (int kk = 0; kk < nk; ++kk) {
    const double uk = u[kk];
    const double *restrict yk = Yb + kk * ld;
#pragma omp simd
    for (int t = 0; t < (int)M; ++t) sc[t] = fma(yk[t], uk, sc[t]);
  }
#endif
}

/* ---- the pass ------------------------------------------------------------- */
typedef struct cpu_problem {
  int64_t n;              /* dimension d */
  const double *U;        /* n x n column-major, upper triangle (truncated factor) */
  const double *a, *b;    /* permuted, scaled bounds */
  int qmc_type;           /* 0 Richtmyer, 1 Sobol */
  const double *q;        /* Richtmyer generators (n-1) */
  const double *shifts;   /* Richtmyer (n-1) x n_reps */
  const uint32_t *V;      /* Sobol (n-1) x 32 */
  int64_t sobol_first;
  const uint64_t *ushifts;/* Sobol (n-1) x n_reps */
  int64_t n_bits;
} cpu_problem;

typedef struct tile_ws {
  double *Y, *S, *c, *dc, *p;
} tile_ws;

static inline int64_t imin64(int64_t x, int64_t y) { return x < y ? x : y; }
static inline int64_t imax64(int64_t x, int64_t y) { return x > y ? x : y; }

/* rand_points! + Phi^-1 for column i (1-based) of the tile:
 * src/qmc_generators.jl:137-204 and src/qmc.jl:385-387 */
static void points_quantiles(const cpu_problem *P, int64_t ld, int64_t n_pass_base, int64_t j1,
                             int64_t len, int64_t i, int64_t k, tile_ws *w) {
  const int64_t n = P->n;
  const double ep0 = DBL_EPSILON, ep1 = 1.0 - DBL_EPSILON, c2 = 1.4142135623730951;
  double *restrict Yc = w->Y + (i - 1) * ld;
  const double *restrict c = w->c;
  const double *restrict dc = w->dc;
  if (P->qmc_type == 0) {
    const double shift = P->shifts[(k - 1) * (n - 1) + (i - 1)];
    const double qi = P->q[i - 1];
    const double base = (double)(n_pass_base + j1); /* point indices stay below 2^53: exact */
    const int nt = (int)len;
#pragma omp simd
    for (int t = 0; t < nt; ++t) {
      double x = (base + (double)t) * qi;
      x = x - floor(x);
      const double u = shift + x;
      Yc[t] = u - (u > 1.0 ? 1.0 : 0.0);
    }
  } else {
    const int L = (int)P->n_bits;
    const uint64_t mask = (L >= 64) ? ~(uint64_t)0 : (((uint64_t)1 << L) - 1);
    const double invscale = ldexp(1.0, -L);
    const uint64_t shift = P->ushifts[(k - 1) * (n - 1) + (i - 1)] & mask;
    const uint32_t *Vi = P->V + (i - 1) * 32;
    /* the generator's integers (Sobol.jl + copyt_as_UInt64!): Gray-code
     * recurrence over the tile's consecutive indices */
    uint64_t idx = (uint64_t)(P->sobol_first + n_pass_base + j1 - 1);
    uint64_t g = idx ^ (idx >> 1);
    uint32_t xi = 0;
    for (int bb = 0; bb < 32; ++bb)
      if ((g >> bb) & 1u) xi ^= Vi[bb];
    for (int64_t t = 0; t < len; ++t) {
      if (t > 0) {
        const uint32_t lo = (uint32_t)(idx + (uint64_t)t);
        if (lo) xi ^= Vi[__builtin_ctz(lo)];
      }
      Yc[t] = (double)((((uint64_t)xi & mask) ^ shift) & mask) * invscale;
    }
  }
  /* tent, affine map into [c, c + dc], clamp, Phi^-1 */
  const int nt = (int)len;
#pragma omp simd
  for (int t = 0; t < nt; ++t) {
    double u = Yc[t];
    u = fabs(fma(u, 2.0, -1.0));
    u = fma(u, dc[t], c[t]);
    u = u < ep0 ? ep0 : u; /* min(max(u, ep0), ep1) of non-NaN u */
    u = u > ep1 ? ep1 : u;
    Yc[t] = c2 * erfinv_v(fma(2.0, u, -1.0));
  }
}

static double dense_tile(const cpu_problem *P, int64_t bi, int64_t bi2, int64_t ld, int64_t n_pass_base,
                         int64_t j1, int64_t len, int64_t k, double c_1, double dc_1, tile_ws *w) {
  const int64_t n = P->n;
  const double *U = P->U;
  const double c2 = 1.4142135623730951;
  double *restrict Y = w->Y;
  double *restrict S = w->S;
  double *restrict c = w->c;
  double *restrict dc = w->dc;
  double *restrict p = w->p;
  /* GEMM rows: the tile's rows rounded up to 8 (rows past len are zeros in Y
   * and are never read back) */
  const int64_t mrows = (len + 7) / 8 * 8;
  for (int64_t t = 0; t < len; ++t) {
    c[t] = c_1;
    dc[t] = dc_1;
    p[t] = dc_1;
  }
  memset(S, 0, sizeof(double) * (size_t)(ld * bi));
  for (int64_t ii1 = 1; ii1 <= n - 1; ii1 += bi) {
    const int64_t ii2 = imin64(ii1 + bi - 1, n - 1);
    if (ii1 > 1) /* S = Y[:, 1:ii1-1] U[1:ii1-1, ii1+1:ii2+1]   (:350-362) */
      gemm(mrows, ii2 - ii1 + 1, ii1 - 1, Y, ld, U + ii1 * n, n, 0.0, S, ld);
    for (int64_t i1 = ii1; i1 <= ii2; i1 += bi2) {
      const int64_t i2 = imin64(i1 + bi2 - 1, ii2);
      if (i1 > ii1) { /* S[:, rest] += Y[:, prev] U[prev, i1+1:ii2+1]   (:367-378) */
        const int64_t prev1 = imax64(ii1, i1 - bi2), prev2 = i1 - 1;
        gemm(mrows, ii2 - i1 + 1, prev2 - prev1 + 1, Y + (prev1 - 1) * ld, ld, U + i1 * n + (prev1 - 1), n, 1.0,
             S + (i1 - ii1) * ld, ld);
      }
      for (int64_t i = i1; i <= i2; ++i) {
        points_quantiles(P, ld, n_pass_base, j1, len, i, k, w);
        /* in-block dot S[:, col] += Y[:, i1:i] U[i1:i, i+1]   (:394-403) */
        double *restrict sc = S + (i - ii1) * ld;
        inblock_dot(mrows, (int)(i - i1 + 1), Y + (i1 - 1) * ld, ld, U + i * n + (i1 - 1), sc);
        /* bounds, CDFs, weight (:405-429) */
        const double a_i = P->a[i], b_i = P->b[i];
        const double inv_u = 1.0 / (U[i * n + i] * c2);
        const int nt = (int)len;
#pragma omp simd
        for (int t = 0; t < nt; ++t) {
          const double s = sc[t];
          double cv = (a_i - s) * inv_u;
          double dv = (b_i - s) * inv_u;
          cv = cv > 9.0 ? 9.0 : cv; /* max(min(x, 9), -9); a = -inf gives -9 */
          cv = cv < -9.0 ? -9.0 : cv;
          dv = dv > 9.0 ? 9.0 : dv;
          dv = dv < -9.0 ? -9.0 : dv;
          cv = erf(cv);
          dv = erf(dv);
          cv = 0.5 * (1.0 + cv);
          dv = 0.5 * (1.0 + dv) - cv;
          c[t] = cv;
          dc[t] = dv;
          p[t] *= dv;
        }
      }
    }
  }
  double sum = 0.0;
  for (int64_t t = 0; t < len; ++t) sum += p[t];
  return sum;
}

/* One qmc_loop! pass (src/qmc.jl:315-444): m points of every shift, folded
 * into the running means qmc_reps (n_reps; pass n_pts0 = 0 for the first
 * pass).  n_pass_base is the generator position of the pass (next_points!).
 * Returns 0, or nonzero when BLAS is not bound or memory runs out. */
int cpu_qmc_pass(const cpu_problem *P, int64_t m, int64_t n_reps, int64_t n_pts0, int64_t n_pass_base,
                 double c_1, double dc_1, int64_t bi, int64_t bi2, int64_t bj, int threads, double *qmc_reps) {
  if (!g_dgemm) return 1;
  const int64_t n = P->n;
  if (n < 2) return 3;
  if (threads <= 0) threads = omp_get_max_threads();
  const int64_t n_tiles = (m + bj - 1) / bj;
  double *tile_sum = (double *)malloc(sizeof(double) * (size_t)n_tiles);
  if (!tile_sum) return 4;
  const int blas_threads = g_get_threads();
  g_set_threads(1);
  int fail = 0;
#pragma omp parallel num_threads(threads)
  {
    tile_ws w;
    const int64_t ld = (bj + 7) / 8 * 8; /* leading dimension: whole 8-row vectors */
    w.Y = (double *)aligned_alloc(64, sizeof(double) * (size_t)(ld * (n - 1) + 8));
    if (w.Y) memset(w.Y, 0, sizeof(double) * (size_t)(ld * (n - 1) + 8));
    w.S = (double *)aligned_alloc(64, sizeof(double) * (size_t)(ld * bi + 8));
    w.c = (double *)aligned_alloc(64, sizeof(double) * (size_t)(3 * ld + 8));
    const int ok = w.Y && w.S && w.c;
    if (!ok) {
#pragma omp atomic write
      fail = 1;
    } else {
      w.dc = w.c + ld;
      w.p = w.c + 2 * ld;
    }
    for (int64_t k = 1; k <= n_reps; ++k) {
#pragma omp for schedule(dynamic, 1)
      for (int64_t tl = 0; tl < n_tiles; ++tl) {
        if (!ok) continue;
        const int64_t j1 = tl * bj + 1, len = imin64(bj, m - tl * bj);
        tile_sum[tl] = dense_tile(P, bi, bi2, ld, n_pass_base, j1, len, k, c_1, dc_1, &w);
      }
#pragma omp single
      {
        double s = 0.0;
        for (int64_t tl = 0; tl < n_tiles; ++tl) s += tile_sum[tl];
        const double inv = 1.0 / (double)(n_pts0 + m);
        const double mean_rep = s * inv;
        const double old_weight = (double)n_pts0 * inv;
        qmc_reps[k - 1] = fma(qmc_reps[k - 1], old_weight, mean_rep);
      }
    }
    free(w.Y);
    free(w.S);
    free(w.c);
  }
  g_set_threads(blas_threads);
  free(tile_sum);
  return fail ? 4 : 0;
}

/* vectorised erfinv of n values (for its unit test) */
void cpu_erfinv(int64_t n, const double *x, double *y) {
#pragma omp simd
  for (int64_t i = 0; i < n; ++i) y[i] = erfinv_v(x[i]);
}

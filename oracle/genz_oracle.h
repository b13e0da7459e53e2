/*
 * genz_oracle.h -- CPU double-precision restatement of the reference's
 * qmc_pnorm! path (JakobPeterlin/DBGenzPaper, Julia).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product is compared against; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  Nothing in
 * dbgenzpaper_b200/ links, includes-for-use or calls it.
 *
 * Conventions: all matrices are column-major (Julia layout), indices in the
 * API are 0-based, perm[] holds 0-based original variable indices.
 *
 * Parity status: the reference cannot run in this container (no Julia), so
 * this restatement is pinned by the reference's own test assertions
 * (test/runtests.jl), by closed-form known answers the reference's scripts
 * use (scripts/simulations/mwp.jl:80-116, temp.jl:40-76) and by the values
 * the reference publishes for the same workloads
 * (data/sims/table_sparse_dense1.tex) -- see tests/test_oracle.py.
 */
#ifndef DBGZ_GENZ_ORACLE_H
#define DBGZ_GENZ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors QMCOpts (src/qmc.jl:15-27); n_blocks is irrelevant here. */
typedef struct orc_opts {
  int64_t chol_block_size;   /* bs1 */
  int64_t chol_block_size2;  /* bs2 */
  int64_t m;                 /* points per pass */
  int64_t block_size_i;
  int64_t block_size_i2;
  int64_t block_size_j;
  int64_t n_reps;            /* number of random shifts */
  int64_t n_bits;            /* Sobol integer grid bits */
  int64_t max_pts;
  double max_abs_err;
} orc_opts;

enum { ORC_RICHTMYER = 0, ORC_SOBOL = 1 };
enum { ORC_CDF_ERF = 0, ORC_CDF_ERFC = 1 };

/* deterministic special functions shared with the GPU factorisation */
double orc_det_erf(double x);
double orc_det_exp(double x);
/* double-precision inverse error function (Newton-refined, libm erf/erfc) */
double orc_erfinv(double x);

/* src/cholesky.jl:445-628.  M (n x n) in/out, a/b in/out (scaled, permuted).
 * Returns rank in *rank. */
void orc_cholesky_genz(int64_t n, double *M, double *a, double *b,
                       int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                       int64_t *perm, double *scale_vec, int64_t *rank);
/* the same, and (when margins is not NULL) for every pivot step i the gap
 * between the winning score and the best other candidate of the panel
 * (diagnostics of near-ties; +inf where the panel has one candidate) */
void orc_cholesky_genz_margins(int64_t n, double *M, double *a, double *b,
                               int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                               int64_t *perm, double *scale_vec, int64_t *rank, double *margins);
/* src/cholesky.jl:244-432 (diagonal pivoting; a, b scaled, not permuted) */
void orc_cholesky_rowmax(int64_t n, double *M, double *a, double *b,
                         int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                         int64_t *perm, double *scale_vec, int64_t *rank);
/* src/cholesky.jl:24-123.  M is nr x n; perm 0-based, permuted in place;
 * k_js (length rank) receives the 1-based block ends, *k_0 the number of
 * zero-level columns moved to the end. */
void orc_adapt_low_rank(int64_t nr, int64_t n, double *M, double *a, double *b, int64_t rank, int64_t *perm,
                        double eps1, int64_t *k_js, int64_t *k_0);
/* src/cholesky.jl:144-242 */
void orc_cholesky_classic(int64_t n, double *M, double *a, double *b,
                          int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                          double *scale_vec);
/* src/qmc.jl:133-142; eps_T = eps(T) of the working type */
void orc_truncate_U(int64_t n, double *U, double eps_T);

/* src/qmc_generators.jl:300-310 and :314-325 */
void orc_sqrt_primes(int64_t n, double *q);
void orc_richtmyer_mat(int64_t m, int64_t n, const double *q, int64_t n0, double *X);
/* Gray-code Sobol integer points: X[j + i*m] = point (first + j), dim i,
 * as the 32-bit grid value floor(x * 2^32).  V is dims x 32 (row per dim). */
void orc_sobol_points(int64_t dims, const uint32_t *V, int64_t first, int64_t m,
                      uint32_t *X);

/* A prepared problem: the output of the QMCData constructor. */
typedef struct orc_problem {
  int64_t n;              /* dimension d */
  const double *U;        /* n x n, upper triangle used */
  const double *a, *b;    /* permuted, scaled bounds (length n) */
  int qmc_type;           /* ORC_RICHTMYER / ORC_SOBOL */
  const double *q;        /* Richtmyer: n-1 generators */
  const double *shifts;   /* Richtmyer: (n-1) x n_reps */
  const uint32_t *V;      /* Sobol: (n-1) x 32 direction numbers */
  int64_t sobol_first;    /* Sobol: index of the first point of pass 0 */
  const uint64_t *ushifts;/* Sobol: (n-1) x n_reps digital shifts */
  int cdf_form;           /* ORC_CDF_ERF (QMCData) / ORC_CDF_ERFC (QMCData_Distributions) */
  int sparse;             /* 1: QMCDataSparse loop over strict-upper CSC */
  int64_t gen_base0;      /* generator position of the first pass (0 for a
                             fresh QMCData; next_points! advances it by m) */
  double *logw;           /* optional (NULL: unused), m x n_reps: each sample's
                             log p = sum of log dc over its variables, of the
                             last pass (a diagnostic; no reference counterpart) */
} orc_problem;

/* src/qmc.jl:783-850 (+ the loops :315-444, :485-608, :618-718).
 * qmc_reps (n_reps) receives the per-shift running means.  threads <= 0
 * means use the OpenMP default. */
void orc_qmc_pnorm(const orc_problem *P, const orc_opts *o, int threads,
                   double *result, double *err, int64_t *n_pts, double *qmc_reps);

#ifdef __cplusplus
}
#endif
#endif

/*
 * dbgenz.h -- C ABI of the B200 Genz QMC multivariate-normal probability
 * library (libdbgenz.so).
 *
 * This is the drop-in boundary for the reference's qmc_pnorm! path
 * (JakobPeterlin/DBGenzPaper, Julia).  Every entry point names the
 * reference function it replaces (file:line in that repository).  A Julia
 * caller binds these with ccall; any C caller can use them directly.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Matrices are column-major (Julia
 *     layout) with leading dimension equal to the row count.
 *   - Host pointers unless the name says _dev.  Every call is synchronous
 *     on the context's own CUDA stream unless it says otherwise.
 *   - Indices are 0-based (perm[i] is the 0-based original variable).
 *   - Every function returns a dbgz_status; nothing throws or aborts across
 *     the ABI.  dbgz_last_error() gives a one-line message for the last
 *     failing call on a context.
 *   - One context per host thread (the reference's QMCData is not reentrant
 *     either, src/qmc.jl:335).  Contexts are independent.
 *   - There is no CPU fallback: without a usable CUDA device dbgz_create
 *     fails with DBGZ_ERR_CUDA.
 */
#ifndef DBGENZ_H
#define DBGENZ_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DBGZ_ABI_VERSION 1

typedef enum dbgz_status {
  DBGZ_OK = 0,
  DBGZ_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad enum, bad size */
  DBGZ_ERR_RANK_DEFICIENT = 2,   /* src/qmc.jl:195-197 ArgumentError */
  DBGZ_ERR_NONFINITE_INPUT = 3,  /* NaN in Sigma, NaN bounds, a > b */
  DBGZ_ERR_DIMENSION = 4,        /* d < 2, or beyond a kernel's limit */
  DBGZ_ERR_OUT_OF_MEMORY = 5,
  DBGZ_ERR_CUDA = 6,             /* CUDA runtime error or no device */
  DBGZ_ERR_TIMEOUT = 7,          /* a bounded device-side wait gave up */
  DBGZ_ERR_UNSUPPORTED = 8       /* mode not available for this problem */
} dbgz_status;

typedef enum dbgz_qmc_type {
  DBGZ_QMC_RICHTMYER = 0, /* RichtmyerQMC, src/qmc_generators.jl:8-13,47-54 */
  DBGZ_QMC_SOBOL = 1      /* SobolQMC,     src/qmc_generators.jl:16-26,57-65 */
} dbgz_qmc_type;

typedef enum dbgz_structure {
  DBGZ_STRUCTURE_DENSE = 0,  /* QMCData:       cholesky_genz!, dense loop  */
  DBGZ_STRUCTURE_SPARSE = 1  /* QMCDataSparse: cholesky_classic!, CSC loop */
} dbgz_structure;

typedef enum dbgz_cdf_form {
  DBGZ_CDF_ERF = 0,  /* QMCData: c = (1 + erf(x))/2            src/qmc.jl:405-429 */
  DBGZ_CDF_ERFC = 1  /* QMCData_Distributions: c = erfc(-x)/2  src/qmc.jl:579-593 */
} dbgz_cdf_form;

typedef enum dbgz_precision {
  /* Double precision everywhere: the reference's Float64 arithmetic. */
  DBGZ_PREC_FP64 = 0,
  /* FP32 special functions and weights (FP64 tail, FP64 weight product
   * and reductions); the conditioning contraction on tcgen05 tensor cores
   * with TF32 operands accumulated in FP32. */
  DBGZ_PREC_FP32_TF32 = 1,
  /* As above with the contraction as three BF16 products (hi*hi + hi*lo +
   * lo*hi of the split operands) accumulated in FP32. */
  DBGZ_PREC_FP32_SPLIT_BF16 = 2,
  /* FP32 numerics of the two modes above with the contraction on CUDA
   * cores (no tensor cores); an ablation of the tensor-core choice. */
  DBGZ_PREC_FP32_SIMT = 3
} dbgz_precision;

/* Mirrors QMCOpts (src/qmc.jl:15-27).  Block sizes that only steer CPU
 * threading (block_size_j, n_blocks) are accepted and ignored; the GPU
 * tiles are chosen by the library. */
typedef struct dbgz_opts {
  int64_t chol_block_size;   /* bs1 of cholesky_genz!/classic! (64)   */
  int64_t chol_block_size2;  /* bs2 (512)                             */
  int64_t m;                 /* QMC points per pass (10^4)            */
  int64_t block_size_i;      /* accepted, unused on the GPU (64)      */
  int64_t block_size_i2;     /* accepted, unused on the GPU (32)      */
  int64_t block_size_j;      /* accepted, unused on the GPU (64)      */
  int64_t n_blocks;          /* accepted, unused on the GPU           */
  int64_t n_reps;            /* random shifts (12)                    */
  int64_t n_bits;            /* Sobol integer grid bits, 1..32 (32)   */
  int64_t max_pts;           /* adaptive stop: points per shift (10^4)*/
  double max_abs_err;        /* adaptive stop: 3*SEM target (1e-6)    */
} dbgz_opts;

typedef struct dbgz_ctx dbgz_ctx;
typedef struct dbgz_problem dbgz_problem;

/* Fills the defaults of QMC_opts(T) (src/qmc.jl:111-125). */
void dbgz_default_opts(dbgz_opts *opts);
const char *dbgz_status_string(int status);
int dbgz_abi_version(void);

/* Context: one CUDA device, one stream, reusable workspaces.  A context
 * caches the device buffers of freed problems and hands them to later
 * problems of similar size (stream-ordered on its stream), so repeated
 * prepare/free cycles make no cudaMalloc/cudaFree calls.  Free every
 * problem of a context before destroying it (DBGZ_ERR_INVALID_ARGUMENT
 * otherwise, and nothing is destroyed).  A context is used by one host
 * thread at a time. */
int dbgz_create(int device, dbgz_ctx **out);
int dbgz_destroy(dbgz_ctx *ctx);
/* Returns the cached buffers of the context to the driver (after waiting
 * for its stream); *freed_bytes (may be NULL) receives their total size.
 * No reference counterpart (the reference runs on host memory). */
int dbgz_release_cached(dbgz_ctx *ctx, uint64_t *freed_bytes);
/* Upper bound on the device bytes of stored forward state (y, s, dc, p s-bar
 * of every sample-variable) that one gradient call may hold; larger sample
 * counts run the forward and adjoint passes in chunks of whole 128-sample
 * tiles (default 48 GiB).  No reference counterpart. */
int dbgz_set_state_budget(dbgz_ctx *ctx, uint64_t bytes);
/* Banded (QMCDataSparse) gradients keep, instead of every sample's forward
 * state, a checkpoint every `segment` dimensions (the band's recent values
 * and the recursion state) and recompute each segment's state from its
 * checkpoint just before the adjoint sweeps it (default 256; 0 stores the
 * whole forward state as the dense path does).  The results are the same
 * bits either way.  No reference counterpart. */
int dbgz_set_grad_checkpoints(dbgz_ctx *ctx, int64_t segment);
const char *dbgz_last_error(const dbgz_ctx *ctx);

/* Device-side timing of the library's own work, measured with CUDA events
 * recorded on the context's stream (the stream every kernel is launched
 * on).  Off by default; costs two event records per launch when on. */
typedef struct dbgz_profile {
  double pnorm_ms;          /* last dbgz_pnorm*: first launch to last copy  */
  double loop_ms;           /* its integration-loop launches, summed        */
  double finalize_ms;       /* its per-shift reduction launches, summed     */
  int64_t loop_launches;    /* integration-loop kernels it launched         */
  int64_t kernel_launches;  /* every kernel it launched                     */
  double prepare_ms;        /* last dbgz_prepare: upload + factorisation    */
  int64_t prepare_launches; /* kernels the last dbgz_prepare launched       */
  double sigma_adjoint_ms;  /* last dbgz_problem_sigma_adjoint              */
  int64_t grad_state_bytes; /* last gradient call: stored forward state     */
  int64_t grad_chunks;      /* last gradient call: sample chunks it ran     */
} dbgz_profile;
int dbgz_set_profiling(dbgz_ctx *ctx, int enable);
int dbgz_get_profile(const dbgz_ctx *ctx, dbgz_profile *out);

/* ---- the qmc_pnorm! path ------------------------------------------- */

/* Constructor of QMCData / QMCDataSparse (src/qmc.jl:149-202, :225-282):
 * copies Sigma (d x d), a, b (length d) to the device, runs the pivoted
 * (dense) or classic (sparse) blocked Cholesky there in FP64, checks the
 * rank (DBGZ_ERR_RANK_DEFICIENT, as the reference's ArgumentError),
 * truncates |U_ij| < eps/(9d) (src/qmc.jl:133-142) and stores the point
 * generator:
 *   Richtmyer: shifts is (d-1) x n_reps doubles in [0,1), the values the
 *              reference draws with rand(rng, T, n-1, n_reps)
 *              (src/qmc_generators.jl:52); ushifts, sobol_* unused.
 *   Sobol:     ushifts is (d-1) x n_reps uint64 digital shifts
 *              (src/qmc_generators.jl:63); sobol_dirnums is (d-1) x 32
 *              direction numbers v_k of each dimension as 32-bit integers
 *              (row per dimension), or NULL for the library's own table
 *              (dbgz_sobol_dirnums); sobol_first is the Gray-code index
 *              (0 = the all-zero point) of the first point of the first
 *              pass: the number of next! calls the caller's SobolSeq has
 *              made, plus one.  SobolQMC's skip(SobolSeq(d), 2m-1) makes
 *              2^floor(log2(2m)) of them (Sobol.jl's skip with exact =
 *              false), so its first point is 2^floor(log2(2m)) + 1.
 * The problem keeps its own generator position: like the reference's
 * QMCData, a second dbgz_pnorm on the same problem continues from the
 * points the previous call ended on (src/qmc.jl:836). */
int dbgz_prepare(dbgz_ctx *ctx, int64_t d, const double *Sigma, const double *a,
                 const double *b, const dbgz_opts *opts, int qmc_type, int structure,
                 int cdf_form, const double *shifts, const uint64_t *ushifts,
                 const uint32_t *sobol_dirnums, int64_t sobol_first,
                 dbgz_problem **out);
int dbgz_problem_free(dbgz_problem *p);

/* Selects the CDF form used by later dbgz_pnorm calls on p.  The
 * reference's QMCData_Distributions(D) (src/qmc.jl:210-215) wraps the same
 * factorisation and generator state as D with the erfc form; a caller
 * switches the form of one problem instead of copying it. */
int dbgz_problem_set_cdf_form(dbgz_problem *p, int cdf_form);

/* Drops the factor's entries more than `bandwidth` above the diagonal
 * (U[l,t] = 0 for t - l > bandwidth) and rebuilds the derived operands.
 * No counterpart in the reference: QMCDataSparse keeps every entry that
 * survives the eps/(9d) truncation (src/qmc.jl:270-272); the banded
 * workload at d = 10^4 (AR(1) covariance, whose factor is dense with
 * geometric decay) specifies this band truncation on top of it. */
int dbgz_problem_truncate_band(dbgz_problem *p, int64_t bandwidth);

/* Reads back the factorisation held by a prepared problem: U (d x d,
 * upper triangle meaningful, as CholeskyGenz.U), perm, permuted and scaled
 * a and b, scale_vec, rank (src/cholesky.jl:5-14).  Any pointer may be
 * NULL. */
int dbgz_problem_factor(const dbgz_problem *p, double *U, int64_t *perm, double *a,
                        double *b, double *scale_vec, int64_t *rank);

/* qmc_pnorm!(D) (src/qmc.jl:783-850): runs passes of m points x n_reps
 * shifts until n_pts >= max_pts or 3*SEM < max_abs_err and returns the
 * mean over shifts, 3*SEM and the number of points per shift.  qmc_reps
 * (length n_reps, may be NULL) receives the per-shift running means. */
int dbgz_pnorm(dbgz_problem *p, int precision, double *result, double *err,
               int64_t *n_pts, double *qmc_reps);

/* Per-sample log-weights of one pass (no reference counterpart: a view of
 * the estimator of qmc_loop!, src/qmc.jl:315-444, whose weight is
 * p = dc_1 dc_2 ... dc_d, src/qmc.jl:405-429).  Runs one pass of m points x
 * n_reps shifts at the problem's current generator position -- the points
 * the next dbgz_pnorm pass would take; the position does not advance -- and
 * writes log p of every sample, the sum of log dc over its variables in
 * FP64, to logw (m x n_reps, column-major: point j of shift k at
 * logw[k * m + j]).  The log-weights stay finite where p underflows to 0
 * (for example 1000 bounds at marginal probabilities 1e-3..1e-1), so the
 * estimate can be compared between precisions in log space.  qmc_reps
 * (n_reps, may be NULL) receives the pass's per-shift means of p. */
int dbgz_pnorm_logw(dbgz_problem *p, int precision, double *logw, double *qmc_reps);

/* dbgz_pnorm with the adaptive loop driven on the device: one CUDA graph
 * launch per call runs every pass -- a conditional while node whose body is
 * one pass and a one-block step that updates the running means, forms the
 * estimate and 3*SEM, advances the point offset and decides on another pass
 * -- with no host round trip between passes.  Same results (bit for bit),
 * generator state and errors as dbgz_pnorm; the graph is kept with the
 * problem for later calls. */
int dbgz_pnorm_graph(dbgz_problem *p, int precision, double *result, double *err,
                     int64_t *n_pts, double *qmc_reps);

/* Gradient of the estimate (no counterpart in the reference).  Runs one
 * pass of m points x n_reps shifts on the problem's current point set (the
 * first pass of dbgz_pnorm; the generator is not advanced), keeps the
 * forward state in device memory, and runs the adjoint of the sequential
 * conditioning on the same points (common random numbers): the returned
 * gradients are exact derivatives of the returned estimate.  The pivot
 * order is held fixed.
 *   dP_da, dP_db: length d, original variable order and scale (NULL skips);
 *   dP_dU: d x d column-major, with respect to the factor U in the
 *          permuted, correlation-scaled coordinates dbgz_problem_factor
 *          returns (upper triangle with the diagonal; NULL skips).
 * Dense structure and erf-form CDF only.  Device memory: four d x N state
 * arrays of the working type (N = samples of the pass) plus partial sums. */
int dbgz_pnorm_grad(dbgz_problem *p, int precision, double *result, double *err,
                    int64_t *n_pts, double *dP_da, double *dP_db, double *dP_dU);

/* dP/dSigma from the outputs of dbgz_pnorm_grad, through the pivoted
 * Cholesky (permutation held fixed) and the correlation scaling of
 * dbgz_prepare; no counterpart in the reference.  dP_dU is the factor
 * gradient (d x d column-major, upper triangle read), dP_da / dP_db the
 * bound gradients in the original order (NULL = zero).  dP_dSigma (d x d
 * column-major, symmetric) is the gradient for symmetric perturbations:
 * dP = sum_ij dP_dSigma[i,j] E[i,j] for symmetric E, so that for
 * Sigma = B B' + diag(psi), dP/dB = 2 dP_dSigma B.  FP64 throughout
 * (cuBLAS TRMM/TRSM/GEMM on the context's stream). */
int dbgz_problem_sigma_adjoint(dbgz_problem *p, const double *dP_dU, const double *dP_da,
                               const double *dP_db, double *dP_dSigma);
/* dbgz_pnorm_grad followed by dbgz_problem_sigma_adjoint with the factor
 * gradient kept on the device: P, its 3 SEM error, dP/da, dP/db (original
 * order, may be NULL) and dP_dSigma (required, as above).  No counterpart in
 * the reference. */
int dbgz_pnorm_grad_sigma(dbgz_problem *p, int precision, double *result, double *err,
                          int64_t *n_pts, double *dP_da, double *dP_db, double *dP_dSigma);

/* ---- allocation-free pass -------------------------------------------
 * No counterpart in the reference.  Some callers cannot let a library
 * allocate device memory: a host framework that owns every device buffer
 * and hands them to the library (an XLA/JAX custom call, a Julia program
 * whose GPU memory is CUDA.jl's pool), or a latency-critical caller for
 * whom cudaMalloc/cudaFree would synchronise the whole device.  For them
 * this entry point runs one FP64 integration pass of qmc_pnorm! (Richtmyer
 * points, erf-form CDF: the loop of src/qmc.jl:315-444 for one pass) and
 * allocates nothing.  Its scratch (per-target constants, per-CTA y
 * workspace, per-tile partial sums) is one fixed 32 MiB array compiled
 * into the library, which every GPU that loads the library holds until
 * the process exits.
 *   Inputs, device pointers: U (d x d truncated factor, column-major, as
 *   dbgz_problem_factor returns it), a and b (permuted, scaled bounds,
 *   length d), q (d-1 lattice generators, dbgz_sqrt_primes), shifts
 *   ((d-1) x n_reps in [0,1]).  n_base is the generator position of the
 *   pass (0 for the first pass, then m, 2m, ...).
 *   Output, device pointer: qmc_reps (n_reps), each shift's mean over its
 *   m points.
 *   stream: a cudaStream_t (NULL: the legacy default stream) on the current
 *   device; the call only enqueues work and returns.
 * Limits: 2 <= d <= 8192 and ceil(m/128) * n_reps <= 131072; larger sizes
 * return DBGZ_ERR_DIMENSION.  Large d runs on fewer CTAs (the workspace
 * share of one CTA grows with d), so this is slower than dbgz_pnorm.
 * The first call in a CUDA context (normally the primary context of each
 * device) looks up the array's device address in that context
 * (cudaGetSymbolAddress) and keeps it, keyed on the context's unique id,
 * so a new context -- also the primary context re-created after
 * cudaDeviceReset -- gets its own look-up; make the first call in each
 * context before any stream capture.  All calls share the one array and leave their
 * intermediate data in it: calls whose work overlaps on the GPU (other
 * streams or host threads at the same time) race and corrupt each other's
 * results, so serialise them. */
int dbgz_pnorm_pass_noalloc(int64_t d, const double *U, const double *a, const double *b,
                            const double *q, const double *shifts, int64_t m, int64_t n_reps,
                            int64_t n_base, double *qmc_reps, void *stream);

/* Many independent problems in one call (QMCData + qmc_pnorm! for each,
 * one pass of opts->m points x opts->n_reps shifts; no reference
 * counterpart, the reference loops over problems on the host).  Problem k
 * has dimension dims[k] (2 <= d <= min(512, chol_block_size2)); Sigma holds
 * the column-major d_k x d_k matrices one after another, a and b the d_k
 * bounds one after another, shifts (Richtmyer) or ushifts (Sobol) the
 * (d_k - 1) x n_reps blocks one after another; sobol_dirnums is one table
 * for the largest d - 1 (NULL: the library's own) and sobol_first the
 * first Sobol index (as in dbgz_prepare).  precision: DBGZ_PREC_FP64 (FP64
 * SIMT loop), DBGZ_PREC_FP32_SIMT, or a tensor-core mode: problems with
 * d - 1 <= 256 then run in the batched tcgen05 loop and the others in the
 * FP32 SIMT loop, as the context's tuning table (dbgz_batch_autotune) or the
 * default (tensor-core loop from d = 25) says.  Inputs are checked on the
 * device (non-finite Sigma, NaN bounds or a > b: DBGZ_ERR_NONFINITE_INPUT;
 * Richtmyer shifts outside [0,1]: DBGZ_ERR_INVALID_ARGUMENT).  results
 * and errs (may be NULL) receive P and 3 SEM per problem, ranks (may be
 * NULL) the Cholesky rank; a problem that is not full rank gets NaN and the
 * call returns DBGZ_ERR_RANK_DEFICIENT after finishing the others. */
int dbgz_pnorm_batch(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const double *Sigma,
                     const double *a, const double *b, const dbgz_opts *opts, int qmc_type,
                     int precision, const double *shifts, const uint64_t *ushifts,
                     const uint32_t *sobol_dirnums, int64_t sobol_first, double *results,
                     double *errs, int64_t *ranks);

/* A reusable batch (the same problems' dimensions, options, generator and
 * precision every run; new Sigma, a, b and shifts each run).  Creation makes
 * the device buffers, tables, tensor maps and kernel configurations and
 * captures one run as a CUDA graph that reads pinned host buffers of the
 * plan: dbgz_batch_plan_buffers returns them (packed as for
 * dbgz_pnorm_batch; shifts are doubles for Richtmyer, uint64 for Sobol), the
 * caller fills them, and each dbgz_batch_plan_run launches the graph (upload,
 * checks, factorisation, loops, reduction, read-back) and waits for it.
 * Results and errors as dbgz_pnorm_batch.  The plan holds its context (like
 * a problem): destroy it before the context. */
typedef struct dbgz_batch_plan dbgz_batch_plan;
int dbgz_batch_plan_create(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims,
                           const dbgz_opts *opts, int qmc_type, int precision,
                           const uint32_t *sobol_dirnums, int64_t sobol_first,
                           dbgz_batch_plan **out);
int dbgz_batch_plan_buffers(dbgz_batch_plan *plan, double **Sigma, double **a, double **b,
                            void **shifts);
int dbgz_batch_plan_run(dbgz_batch_plan *plan, double *results, double *errs, int64_t *ranks);
int dbgz_batch_plan_info(const dbgz_batch_plan *plan, int64_t *n_tensor_problems,
                         int64_t *n_simt_items, int64_t *kernels_per_run, int64_t *host_bytes);
int dbgz_batch_plan_destroy(dbgz_batch_plan *plan);

/* Autotuner of the batch loops: for dimension buckets of 2..512, times the
 * SIMT loop with work items of 256, 1024 and 4096 tile-dimensions and (in
 * the tensor-core precisions, d - 1 <= 256) the batched tensor-core loop on
 * pilot batches of the options' point and shift counts, and stores the
 * fastest choice per dimension in the context (used by later batch calls and
 * plans of this precision and generator).  engine_out and item_dims_out (may
 * be NULL) receive the table, indexed by d = 0..512 (1 = tensor-core loop).
 * dbgz_batch_tuning reads the table in use (the default when not tuned). */
int dbgz_batch_autotune(dbgz_ctx *ctx, int precision, int qmc_type, const dbgz_opts *opts,
                        int32_t *engine_out, int32_t *item_dims_out);
int dbgz_batch_tuning(const dbgz_ctx *ctx, int precision, int qmc_type, int32_t *engine_out,
                      int32_t *item_dims_out, int *tuned);

/* ---- primitives of the path (device compute, host buffers) ---------- */

/* cholesky_genz!(M, a, b, bs1, bs2, bs3, bs4) (src/cholesky.jl:445-628):
 * in place on M (d x d), a, b.  perm (d), scale_vec (d) and rank are
 * outputs.  Pivot choices are made with the library's deterministic FP64
 * erf/exp, so the permutation is reproducible bit for bit. */
int dbgz_cholesky_genz(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b,
                       int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                       int64_t *perm, double *scale_vec, int64_t *rank);
/* cholesky_classic!(M, a, b, bs1..bs4) (src/cholesky.jl:144-242). */
int dbgz_cholesky_classic(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b,
                          int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4,
                          double *scale_vec);

/* cholesky_rowmax!(M, a, b, bs1, bs2, bs3, bs4) (src/cholesky.jl:244-432):
 * Cholesky with diagonal pivoting (the largest remaining diagonal of the
 * bs2 panel, first on ties) on the GPU, with cholesky_genz!'s block
 * structure and arithmetic contract.  Host arrays in/out as in
 * dbgz_cholesky_genz: M (d x d, correlation-scaled then factored in place,
 * upper triangle = U), a and b scaled by 1/sqrt(Sigma_ii) but not permuted
 * (as the reference leaves them), perm (0-based), scale_vec, and rank: the
 * first row whose remaining diagonal is not positive (d when none).  Not
 * called by qmc_pnorm!. */
int dbgz_cholesky_rowmax(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b, int64_t bs1,
                         int64_t bs2, int64_t bs3, int64_t bs4, int64_t *perm, double *scale_vec,
                         int64_t *rank);

/* adapt_low_rank!(M, a, b, rank, perm, eps1) (src/cholesky.jl:24-123):
 * for a factor of rank r (M: nr x n, column-major; columns r+1..n hold the
 * dependent variables' coefficients in rows 1..r), every dependent column
 * with no entry above eps1 in rows 1..r moves to the end; every other is
 * scaled by its last such entry (its level i_j; a and b are scaled with it
 * and swapped when that entry is negative) and placed at the end of the
 * block of level i_j.  Host arrays, updated in place: M, a, b, perm
 * (0-based indices).  k_js (length rank) receives the blocks' 1-based end
 * positions and *k_0 the number of columns moved to the end.  The levels are
 * found on the device and the columns written to their final places by one
 * gather; the values are the reference's. */
int dbgz_adapt_low_rank(dbgz_ctx *ctx, int64_t nr, int64_t n, double *M, double *a, double *b,
                        int64_t rank, int64_t *perm, double eps1, int64_t *k_js, int64_t *k_0);
/* get_sqrt_primes!(q) (src/qmc_generators.jl:300-310), host only. */
int dbgz_sqrt_primes(int64_t n, double *q);
/* richtmyer_mat!(X, q, n0) (src/qmc_generators.jl:314-325): X is m x n
 * doubles, X[i,j] = frac((n0 + i + 1) q_j) computed in FP64. */
int dbgz_richtmyer_mat(dbgz_ctx *ctx, int64_t m, int64_t n, const double *q, int64_t n0,
                       double *X);
/* sobol_mat! + copyt_as_UInt64! (src/qmc_generators.jl:331-352) on the
 * 32-bit grid: X is m x dims uint32, X[j,i] = floor(x_{first+j,i} 2^32)
 * of the Gray-code Sobol sequence with direction numbers V (dims x 32). */
int dbgz_sobol_mat(dbgz_ctx *ctx, int64_t m, int64_t dims, const uint32_t *V,
                   int64_t first, uint32_t *X);
/* The library's own direction numbers (host only): dimension 0 is the
 * van der Corput sequence; dimension i >= 1 uses the i-th primitive
 * polynomial over GF(2) (ordered by degree, then value) with odd initial
 * values m_k < 2^k drawn from a fixed-seed generator (Bratley-Fox
 * construction).  V is dims x 32, V[i*32 + k] = m_{k+1} << (31 - k). */
int dbgz_sobol_dirnums(int64_t dims, uint32_t *V);

#ifdef __cplusplus
}
#endif
#endif /* DBGENZ_H */

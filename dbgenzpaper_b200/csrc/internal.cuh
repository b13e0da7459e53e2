// internal.cuh -- shared declarations of libdbgenz (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstdarg>
#include <map>
#include <string>
#include <vector>

#include "../../include/dbgenz.h"

#define DBGZ_CUDA_TRY(ctx, call)                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return dbgz_fail((ctx), DBGZ_ERR_CUDA, "%s failed: %s (%s:%d)", #call,        \
                       cudaGetErrorString(e_), __FILE__, __LINE__);                 \
  } while (0)

#define DBGZ_TRY(call)                \
  do {                                \
    int s_ = (call);                  \
    if (s_ != DBGZ_OK) return s_;     \
  } while (0)

struct dbgz_ctx;
// A device buffer of the library.  Buffers taken from a context's pool go
// back to it on release (owner set); bytes is the block's capacity.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  dbgz_ctx *owner = nullptr;
};

// Batch engine choices per dimension (dbgz_batch_autotune): engine[d] = 1
// for the tensor-core loop, 0 for the SIMT loop; item_dims[d] = size of the
// SIMT loop's work items in tile-dimensions.
constexpr int64_t kBatchMaxD = 512;
struct BatchTuning {
  bool tuned = false;
  int8_t engine[kBatchMaxD + 1] = {};
  int32_t item_dims[kBatchMaxD + 1] = {};
};

struct dbgz_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  int *d_status = nullptr;  // device-side error word written by bounded waits
  bool profiling = false;
  cudaEvent_t ev[6] = {};   // 0/1: call bracket, 2/3: loop launch, 4/5: finalize
  dbgz_profile prof{};
  int64_t launch_count = 0; // kernels launched by the library on this context
  // Stream-ordered block cache: released buffers wait here for the next
  // request of similar size.  Every user of a block enqueues on `stream`, so
  // a block handed out again is only touched after the work of its previous
  // user; nothing is returned to the driver before dbgz_release_cached or
  // dbgz_destroy (or an allocation failure, which empties the cache and
  // retries once).
  std::multimap<size_t, void *> pool;
  size_t pool_bytes = 0;
  int64_t live_problems = 0;  // problems created on this context and not yet freed
  size_t state_budget = size_t(48) << 30;  // bytes of stored forward state a gradient call may hold
  // banded gradients: dimensions per checkpoint segment (0: store the whole
  // forward state instead)
  int64_t grad_ckpt_seg = 256;
  BatchTuning batch_tune[4][2];            // [precision][qmc_type]
};

// Counts a kernel launch of the library (for dbgz_profile).
inline void dbgz_count_launch(dbgz_ctx *ctx, int n = 1) { ctx->launch_count += n; }

int dbgz_fail(dbgz_ctx *ctx, int status, const char *fmt, ...);
int dbgz_ensure(dbgz_ctx *ctx, DevBuf &b, size_t bytes);
void dbgz_release(DevBuf &b);

// Parameters of one target dimension t (variable t, 0-based) of the loop:
// the lower/upper bound and 1/(U[t,t] sqrt 2).
struct TargetParams64 {
  double a, b, inv_u;
};
struct TargetParams32 {
  float a, b, inv_u, pad;
};

struct dbgz_problem {
  dbgz_ctx *ctx = nullptr;
  int64_t d = 0;
  dbgz_opts opts{};
  int qmc_type = 0, structure = 0, cdf_form = 0;
  int64_t rank = 0;
  // factorisation (device, FP64)
  DevBuf U, a, b, perm, scale;
  // generator (device)
  DevBuf q, shifts, shifts32, V, ushifts;
  int64_t sobol_first = 0;
  int64_t gen_base = 0;  // offset of the current point block (next_points! state)
  // device-driven adaptive loop (driver_graph.cu): a graph per precision and
  // the buffers and constants it was captured with
  cudaGraph_t drv_graph[4] = {};
  cudaGraphExec_t drv_exec[4] = {};
  std::vector<uint64_t> drv_sig[4];
  DevBuf drv_state;
  // derived operands (device, built on first use)
  DevBuf tgt64, tgt32, U32;
  DevBuf Uhi, Ulo, Utf;  // tensor-core operands of the contraction
  int64_t ldU = 0;       // padded leading dimension of Uhi/Ulo/Utf
  // the same for the anti-transposed factor Ub[i, j] = U[d-1-j, d-1-i]
  // (coefficients of the adjoint recurrence, policies.cuh)
  DevBuf Ub, Ub32, Ubhi, Ublo, Ubtf;
  int64_t ldUb = 0;
  DevBuf grad_buf;       // forward state and partial gradients of dbgz_pnorm_grad
  // sparse (banded) structure: CSC of the strict upper factor
  DevBuf csc_colptr, csc_row, csc_val64, csc_val32;
  DevBuf cscb_colptr, cscb_row, cscb_val64, cscb_val32;  // CSC of the anti-transposed factor (adjoint)
  int64_t bandwidth_b = 1;
  int64_t nnz = 0, bandwidth = 0, band = 0;  // band > 0: entries beyond it dropped
  // workspaces
  DevBuf yws, partials, reps;
  double c1 = 0, dc1 = 0;
  bool c1_ready = false;
  // every lower bound is -inf: the forward loops take the one-sided step
  // (dbgz::StepFp64LowerInf / StepFp32LowerInf, the same bits)
  bool lower_inf = false;
};

// ---- factorisation (chol.cu) -------------------------------------------
int dbgz_chol_genz_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b, int64_t bs1,
                       int64_t bs2, int64_t bs3, int64_t bs4, int64_t *perm, double *scale,
                       int64_t *rank_host);
int dbgz_chol_rowmax_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b, int64_t bs1, int64_t bs2,
                         int64_t bs3, int64_t bs4, int64_t *perm, double *scale, int64_t *rank_host);
int dbgz_chol_classic_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b,
                          int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4, double *scale);
int dbgz_truncate_dev(dbgz_ctx *ctx, int64_t n, double *U, double eps_T);
int dbgz_make_targets(dbgz_problem *p);
int dbgz_band_dev(dbgz_ctx *ctx, int64_t d, double *U, int64_t band);
int dbgz_make_U32(dbgz_problem *p);
int dbgz_make_Ub(dbgz_problem *p);

// ---- points (points.cu) --------------------------------------------------
int dbgz_richtmyer_dev(dbgz_ctx *ctx, int64_t m, int64_t n, const double *q, int64_t n0,
                       double *X);
int dbgz_sobol_dev(dbgz_ctx *ctx, int64_t m, int64_t dims, const uint32_t *V, int64_t first,
                   uint32_t *X);

// ---- integration loop (loop_simt.cu) ---------------------------------------
// Which sequential step the loops run (policies.cuh).
// kLoopLogWeight: a forward pass that also writes each sample's log-weight
// log p = log dc_0 + ... + log dc_{d-1} to pa.grad.p (one double per sample,
// [tile * 128 + row]), finite where p itself underflows
enum LoopKind { kLoopForward = 0, kLoopForwardStore = 1, kLoopAdjoint = 2, kLoopLogWeight = 3 };

// Forward state kept for the adjoint and the adjoint's outputs (device
// arrays; element type float or double per precision).
struct GradArrays {
  int64_t N = 0;  // samples of the pass (n_tiles * 128)
  void *y = nullptr, *s = nullptr, *dc = nullptr, *sbar = nullptr;
  double *p = nullptr, *ga = nullptr, *gb = nullptr, *gu = nullptr;
  double dc1 = 0.0;
};

struct PassArgs {
  int kind = kLoopForward;
  GradArrays grad;
  int64_t d;
  int64_t m;          // points per pass
  int64_t n_reps;
  int64_t gen_base;   // Richtmyer: n_base; Sobol: offset added to sobol_first
  int64_t sobol_first;
  int n_bits;
  int qmc_type;
  int cdf_form;
  double c1, dc1;
  int64_t tile0 = 0;  // run tiles [tile0, n_tiles) only (sample chunks of the adjoint)
  const int64_t *gen_base_dev = nullptr;  // device copy of gen_base (device-driven passes)
  bool setup_only = false;  // make the launch's buffers and operands, launch nothing
  // dimension segments (banded loop only, grad.cu): the pass runs the
  // y-indices [i_begin, i_end) (i_end < 0: all); with ck_load it first restores
  // each sample's ring of recent values and recursion state from ck_in; with
  // ck_save = 1 it saves them before every y-index that is a multiple of
  // ck_seg (slot index / ck_seg - 1), with ck_save = 2 once after i_end - 1
  // (slot 0); per slot: ring [W][ck_N] of the pass's value type, state
  // [4][ck_N] doubles.  tile_finish = 0 skips the per-tile end terms and sums.
  int64_t i_begin = 0, i_end = -1;
  int ck_load = 0, ck_save = 0, tile_finish = 1;
  const void *ck_in_ring = nullptr;
  const double *ck_in_state = nullptr;
  void *ck_ring = nullptr;
  double *ck_state = nullptr;
  int64_t ck_seg = 0, ck_N = 0;
  int64_t io_row0 = 0, io_rows = 0;  // rows of the stored-state arrays (0: all d from row 0)
  int store_p = 0;
};
int dbgz_loop_simt(dbgz_problem *p, const PassArgs &pa, int precision, double *partials,
                   int64_t n_tiles);
int dbgz_loop_umma(dbgz_problem *p, const PassArgs &pa, int precision, double *partials,
                   int64_t n_tiles);
// Forward tensor-core loop over many problems of at most two halves (d - 1 <= 256) in
// one launch (batch.cu).  Host tables cover all problems of the batch;
// `probs` lists the ones to run here, largest first.  Device pointers: FP64
// factors (dM + off2[k]), FP32 factors, FP32 targets, 3 first-dimension
// constants per problem, generator data (shifts at offs[k]) and partial sums
// (dpart + part_off[k]).  Resets ctx->d_status; the caller reads it.
struct UmmaBatchArgs {
  int qmc_type = 0, n_bits = 32;
  int64_t m = 0, n_reps = 0, tiles_per_shift = 0, sobol_first = 0;
  std::vector<int64_t> probs;
  const int64_t *dims = nullptr, *off2 = nullptr, *off1 = nullptr, *offs = nullptr, *part_off = nullptr;
  const double *dM = nullptr, *dfirst = nullptr, *dq = nullptr;
  const float *dU32 = nullptr, *dsh32 = nullptr;
  const TargetParams32 *dt32 = nullptr;
  const uint32_t *dV = nullptr;
  const uint64_t *dush = nullptr;
  double *dpart = nullptr;
};
// Tensor-core part of a batch plan: the U^T panels, per-problem descriptors
// (tensor maps of the plan's fixed buffers) and the item list, set up once;
// enqueue issues the panel conversion, the status reset and the loop on
// ctx->stream (no allocation, no host synchronisation: capturable).
struct UmmaBatchPlan {
  dbgz_ctx *ctx = nullptr;
  int mode = 0, qmc_type = 0;
  DevBuf buf;
  char *pan0 = nullptr, *pan1 = nullptr, *d_desc = nullptr;
  int64_t nsel = 0, n_items = 0, grid = 0;
  int smem = 0;
  int64_t *d_dims = nullptr, *d_off2 = nullptr, *d_ld = nullptr, *d_pan = nullptr;
  int32_t *d_iprob = nullptr, *d_itile = nullptr;
  const double *dM = nullptr;
};
int dbgz_umma_batch_setup(dbgz_ctx *ctx, int precision, const UmmaBatchArgs &A, UmmaBatchPlan **out);
int dbgz_umma_batch_enqueue(UmmaBatchPlan *B);
void dbgz_umma_batch_free(UmmaBatchPlan *B);
int dbgz_loop_sparse(dbgz_problem *p, const PassArgs &pa, int precision, double *partials,
                     int64_t n_tiles);
int dbgz_build_csc(dbgz_problem *p);
void dbgz_drop_graphs(dbgz_problem *p);
// dU[t*d + l] (+)= sum_n Y(l, n) S(t, n) over the nc samples, for l < t only,
// Y and S tile-major ([tile][row < d][128 samples], the FP32 layout of
// GradIO) (du_gemm.cu: tcgen05 TF32, split over samples, fixed-order sum of
// the splits).  work: scratch taken from the context's pool.
int dbgz_du_gemm_tf32(dbgz_ctx *ctx, int64_t d, const float *Y, const float *S, int64_t nc, float *dU,
                      bool accumulate, DevBuf &work);
int dbgz_finalize_pass(dbgz_problem *p, const double *partials, int64_t tiles_per_shift,
                       int64_t n_pts0, int64_t m, double *reps);

// grad.cu -- dbgz_pnorm_grad: the estimate and its adjoint on one point set.
//
// No counterpart in the reference (it has no gradient).  One pass of m
// points x n_reps shifts runs the forward loop with the STORE policy
// (y_l, s_t, dc_t and p of every sample kept in HBM, [index][sample]), then
// the same loop kernel runs the adjoint recurrence on the anti-transposed
// factor (policies.cuh).  Per-variable terms (dP/da_t, dP/db_t, dP/dU_tt)
// come out as per-(tile, warp) partial sums reduced here in a fixed order;
// the off-diagonal dP/dU[l, t] = mean over samples of y_l * (p sbar_t) is one
// GEMM of the two stored arrays over the strict upper triangle l < t (FP64:
// dense64.cuh on CUDA cores, split over samples with the split sums added in
// a fixed order; FP32 paths: tcgen05 TF32 with FP32 accumulation, du_gemm.cu).
#include <algorithm>
#include <cmath>
#include <vector>

#include "dense64.cuh"
#include "internal.cuh"

namespace {

// Fixed-order sums of the per-(tile, warp) partial rows part[row * d + t]:
// stage 1 sums `chunk` consecutive rows per CTA column (coalesced over t),
// stage 2 sums the chunk sums in chunk order.
constexpr int kRedChunks = 256;
__global__ void k_reduce_rows(const double *ga, const double *gb, const double *gu, int64_t rows, int64_t d,
                              int64_t chunk, double *csum) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= d) return;
  const int64_t r0 = blockIdx.y * chunk, r1 = r0 + chunk < rows ? r0 + chunk : rows;
  double a = 0.0, b = 0.0, u = 0.0;
  for (int64_t r = r0; r < r1; ++r) {
    a += ga[r * d + t];
    b += gb[r * d + t];
    u += gu[r * d + t];
  }
  double *o = csum + (int64_t)blockIdx.y * 3 * d;
  o[t] = a;
  o[d + t] = b;
  o[2 * d + t] = u;
}
__global__ void k_reduce_chunks(const double *csum, int64_t n_chunks, int64_t d, double *out, int accumulate) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // i in [0, 3d)
  if (i >= 3 * d) return;
  double v = 0.0;
  for (int64_t c = 0; c < n_chunks; ++c) v += csum[c * 3 * d + i];
  out[i] = accumulate ? out[i] + v : v;
}

// Device-side assembly of the outputs: dU64 (d x d FP64, factor coordinates;
// skipped when null), da/db in the original order and scale.  gemm[t*d + l] = sum_n y_l (p sbar_t).
__global__ void k_grad_assemble(const void *gemm, int esz, const double *sums, const int64_t *perm,
                                const double *scale, double inv, int64_t d, double *dU64, double *da, double *db) {
  const int64_t t = blockIdx.y;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; dU64 && l < d;
       l += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (l < t) {
      const size_t ix = (size_t)t * d + l;
      v = (esz == 8 ? static_cast<const double *>(gemm)[ix] : (double)static_cast<const float *>(gemm)[ix]) * inv;
    } else if (l == t) {
      v = sums[2 * d + t] * inv;
    }
    dU64[t * d + l] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int64_t o = perm[t];
    da[o] = sums[t] * inv / scale[o];
    db[o] = sums[d + t] * inv / scale[o];
  }
}

}  // namespace


extern "C" int dbgz_first_dim_cdf(dbgz_problem *p);  // api.cu

int dbgz_sigma_adjoint_dev(dbgz_problem *p, const double *dU, const double *da, const double *db,
                           double *host_out);  // chol_adjoint.cu

static int grad_impl(dbgz_problem *p, int precision, double *result, double *err, int64_t *n_pts, double *dP_da,
                     double *dP_db, double *dP_dU, double *dP_dSigma) {
  if (!p || !result || !err || !n_pts) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_grad: bad precision %d", precision);
  const bool sparse = p->structure == DBGZ_STRUCTURE_SPARSE;
  if (sparse && (dP_dU || dP_dSigma))
    return dbgz_fail(ctx, DBGZ_ERR_UNSUPPORTED, "pnorm_grad: the banded path gives dP/da and dP/db only");
  if (p->cdf_form != DBGZ_CDF_ERF && !sparse)
    return dbgz_fail(ctx, DBGZ_ERR_UNSUPPORTED, "pnorm_grad: the adjoint is built for the erf-form CDF");
  cudaSetDevice(ctx->device);
  const dbgz_opts &o = p->opts;
  const int64_t d = p->d, m = o.m, n_reps = o.n_reps;
  const int64_t tps = (m + 127) / 128, n_tiles = tps * n_reps;
  const size_t esz = precision == DBGZ_PREC_FP64 ? 8 : 4;
  DBGZ_TRY(dbgz_first_dim_cdf(p));
  if (precision != DBGZ_PREC_FP64 && !p->U32.p && !sparse) DBGZ_TRY(dbgz_make_U32(p));
  if (!p->Ub.p) DBGZ_TRY(dbgz_make_Ub(p));
  // Banded problems with dimension checkpoints (ctx->grad_ckpt_seg > 0): the
  // forward pass keeps, every `seg` y-indices, each sample's ring of the last
  // W values and its recursion state (a checkpoint), and the adjoint then
  // runs segment by segment from the last: the segment's y, s, dc recomputed
  // from its checkpoint into a buffer of seg + 2 rows, the adjoint steps of
  // the segment's variables on it, the adjoint's own ring and state carried
  // to the next segment.  The same kernels and arithmetic as storing
  // everything: the same bits, with the stored state of K = ceil((d-1)/seg)
  // checkpoints instead of d rows.
  const int64_t seg = sparse ? ctx->grad_ckpt_seg : 0;
  const int64_t nY = d - 1, K = seg > 0 ? (nY + seg - 1) / seg : 0;
  const bool ckpt = seg > 0 && K >= 1;
  int64_t Wf = 0, Wb = 0;  // ring sizes of the forward and adjoint banded loops
  if (ckpt) {
    PassArgs sa{};
    sa.d = d;
    sa.m = m;
    sa.n_reps = n_reps;
    sa.qmc_type = p->qmc_type;
    sa.n_bits = (int)o.n_bits;
    sa.setup_only = true;
    sa.kind = kLoopAdjoint;  // builds both CSCs
    DBGZ_TRY(dbgz_loop_sparse(p, sa, precision, nullptr, 1));
    Wf = p->bandwidth + 1;
    Wb = p->bandwidth_b + 1;
  }
  const int64_t ck_rows = seg + 2;  // rows of a segment's recomputed state
  // samples per chunk: as many whole tiles as the context's state budget
  // allows (forward-store, adjoint, reduction and the dU GEMM run per chunk;
  // the GEMM accumulates across chunks)
  const size_t state_per_sample =
      ckpt ? (size_t)(K - 1) * (Wf * esz + 32) + (Wb * esz + 32) + 3 * ck_rows * esz
           : (sparse ? 3 : 4) * esz * (size_t)d;
  const size_t tile_bytes = 128 * (state_per_sample + 8) + 3 * 4 * 8 * (size_t)d;
  const int64_t chunk =
      std::max<int64_t>(1, std::min<int64_t>(n_tiles, (int64_t)(ctx->state_budget / tile_bytes)));
  const int64_t N = chunk * 128;
  ctx->prof.grad_state_bytes = (int64_t)(state_per_sample * (size_t)N);
  ctx->prof.grad_chunks = (n_tiles + chunk - 1) / chunk;
  // one allocation: y, s, dc (+ p sbar on the dense path; a segment's rows
  // with checkpoints), checkpoints, p, 3 partial arrays, sums, dU
  const size_t arr = esz * (size_t)(ckpt ? ck_rows : d) * N;
  const size_t ck_bytes = ckpt ? (size_t)(K - 1) * ((size_t)Wf * esz + 32) * N + ((size_t)Wb * esz + 32) * N : 0;
  const size_t part = sizeof(double) * (size_t)chunk * 4 * d;
  const size_t total = (sparse ? 3 : 4) * arr + ck_bytes + 8 * 256 + 8 * (size_t)N + 3 * part +
                       3 * 8 * (size_t)d * (kRedChunks + 1) +
                       (sparse ? 0 : esz * (size_t)d * d + 8 * (size_t)d * d) + 2 * 8 * (size_t)d +
                       8 * (size_t)n_tiles + 16384;
  DBGZ_TRY(dbgz_ensure(ctx, p->grad_buf, total));
  char *base = (char *)p->grad_buf.p;
  auto take = [&](size_t bytes) {
    char *r = base;
    base += (bytes + 255) & ~size_t(255);
    return r;
  };
  GradArrays ga;
  ga.N = N;
  ga.y = take(arr);
  ga.s = take(arr);
  ga.dc = take(arr);
  ga.sbar = sparse ? nullptr : take(arr);
  // checkpoints: slots 0..K-2 (forward: ring [Wf][N], state [4][N]) and the
  // adjoint's carry (ring [Wb][N], state [4][N])
  char *ck_ring = ckpt ? take((size_t)(K > 1 ? K - 1 : 1) * Wf * esz * N) : nullptr;
  double *ck_state = ckpt ? (double *)take((size_t)(K > 1 ? K - 1 : 1) * 32 * N) : nullptr;
  char *cr_ring = ckpt ? take((size_t)Wb * esz * N) : nullptr;
  double *cr_state = ckpt ? (double *)take((size_t)32 * N) : nullptr;
  ga.p = (double *)take(8 * (size_t)N);
  ga.ga = (double *)take(part);
  ga.gb = (double *)take(part);
  ga.gu = (double *)take(part);
  ga.dc1 = p->dc1;
  double *sums = (double *)take(3 * 8 * (size_t)d);
  double *csum = (double *)take(3 * 8 * (size_t)d * kRedChunks);
  void *dU = sparse ? nullptr : take(esz * (size_t)d * d);
  double *dU64 = sparse ? nullptr : (double *)take(8 * (size_t)d * d);
  double *da_o = (double *)take(8 * (size_t)d), *db_o = (double *)take(8 * (size_t)d);
  // the adjoint pass writes per-tile values too (zeros); keep them away from
  // the forward pass's tile sums, which are reduced after the last chunk
  double *adj_tiles = (double *)take(8 * (size_t)n_tiles);
  if (!sparse && precision == DBGZ_PREC_FP64) {
    // rows the passes leave unwritten (y row d-1, sbar row 0) enter the DGEMM:
    // clear them (the FP32 GEMM computes l < t only, which never reads them)
    DBGZ_CUDA_TRY(ctx, cudaMemsetAsync((char *)ga.y + esz * (size_t)(d - 1) * N, 0, esz * N, ctx->stream));
    DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ga.sbar, 0, esz * N, ctx->stream));
  }

  DBGZ_TRY(dbgz_ensure(ctx, p->partials, sizeof(double) * n_tiles));
  DBGZ_TRY(dbgz_ensure(ctx, p->reps, sizeof(double) * n_reps));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(p->reps.p, 0, sizeof(double) * n_reps, ctx->stream));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  const bool prof = ctx->profiling;
  const int64_t launches0 = ctx->launch_count;
  if (prof) cudaEventRecord(ctx->ev[0], ctx->stream);

  PassArgs pa{};
  pa.d = d;
  pa.m = m;
  pa.n_reps = n_reps;
  pa.sobol_first = p->sobol_first;
  pa.n_bits = (int)o.n_bits;
  pa.qmc_type = p->qmc_type;
  pa.cdf_form = p->cdf_form;
  pa.c1 = p->c1;
  pa.dc1 = p->dc1;
  pa.gen_base = p->gen_base;
  pa.grad = ga;
  const bool tensor = !sparse && (precision == DBGZ_PREC_FP32_TF32 || precision == DBGZ_PREC_FP32_SPLIT_BF16);
  auto run = [&](int kind, int64_t t0, int64_t t1) -> int {
    pa.kind = kind;
    pa.tile0 = t0;
    double *tiles = kind == kLoopAdjoint ? adj_tiles : (double *)p->partials.p;
    if (sparse) return dbgz_loop_sparse(p, pa, precision, tiles, t1);
    if (tensor) return dbgz_loop_umma(p, pa, precision, tiles, t1);
    return dbgz_loop_simt(p, pa, precision, tiles, t1);
  };
  // a pass of the banded loop with the segment fields of pa as they stand
  auto sparse_run = [&](int kind, int64_t t0, int64_t t1) -> int {
    pa.kind = kind;
    pa.tile0 = t0;
    double *tiles = kind == kLoopAdjoint ? adj_tiles : (double *)p->partials.p;
    return dbgz_loop_sparse(p, pa, precision, kind == kLoopForwardStore ? adj_tiles : tiles, t1);
  };
  const bool want_U = dP_dU || dP_dSigma;
  DevBuf du_work;  // split partial tiles of the FP32 dU GEMM (back to the pool at the end, stream-ordered)
  struct Release {
    DevBuf &b;
    ~Release() { dbgz_release(b); }
  } release_du{du_work};
  for (int64_t t0 = 0; t0 < n_tiles; t0 += chunk) {
    const int64_t t1 = std::min(n_tiles, t0 + chunk);
    if (!ckpt) {
      // forward keeping the state, then the adjoint on the anti-transposed factor
      DBGZ_TRY(run(kLoopForwardStore, t0, t1));
      DBGZ_TRY(run(kLoopAdjoint, t0, t1));
    } else {
      // forward with checkpoints (and the tile sums of the estimate)
      pa.store_p = 1;
      pa.ck_save = 1;
      pa.ck_ring = ck_ring;
      pa.ck_state = ck_state;
      pa.ck_seg = seg;
      pa.ck_N = N;
      DBGZ_TRY(run(kLoopForward, t0, t1));
      pa.store_p = 0;
      pa.ck_save = 0;
      for (int64_t sg = K - 1; sg >= 0; --sg) {
        // recompute the segment: steps [seg sg, seg (sg + 1)] (one past the
        // segment: s and dc of its last variable come from the next step)
        pa.i_begin = seg * sg;
        pa.i_end = std::min(seg * (sg + 1) + 1, nY);
        pa.ck_load = sg > 0;
        pa.ck_in_ring = ck_ring + (size_t)(sg > 0 ? sg - 1 : 0) * Wf * esz * N;
        pa.ck_in_state = ck_state + (size_t)(sg > 0 ? sg - 1 : 0) * 4 * N;
        pa.io_row0 = seg * sg;
        pa.io_rows = ck_rows;
        pa.tile_finish = 0;
        pa.kind = kLoopForwardStore;
        pa.tile0 = t0;
        DBGZ_TRY(sparse_run(kLoopForwardStore, t0, t1));
        // the adjoint steps of variables seg sg + 1 .. min(seg (sg + 1), d - 1)
        pa.i_begin = nY - std::min(seg * (sg + 1), nY);
        pa.i_end = nY - seg * sg;
        pa.ck_load = sg < K - 1;
        pa.ck_in_ring = cr_ring;
        pa.ck_in_state = cr_state;
        pa.ck_save = sg > 0 ? 2 : 0;
        pa.ck_ring = cr_ring;
        pa.ck_state = cr_state;
        pa.tile_finish = sg == 0;
        DBGZ_TRY(sparse_run(kLoopAdjoint, t0, t1));
        pa.ck_save = 0;
        pa.ck_ring = ck_ring;
        pa.ck_state = ck_state;
      }
      pa.i_begin = 0;
      pa.i_end = -1;
      pa.ck_load = 0;
      pa.io_row0 = 0;
      pa.io_rows = 0;
      pa.tile_finish = 1;
    }
    const int64_t rows = (t1 - t0) * 4, per = (rows + kRedChunks - 1) / kRedChunks;
    const int64_t n_chunks = (rows + per - 1) / per;
    k_reduce_rows<<<dim3((unsigned)((d + 127) / 128), (unsigned)n_chunks), 128, 0, ctx->stream>>>(
        ga.ga, ga.gb, ga.gu, rows, d, per, csum);
    dbgz_count_launch(ctx);
    k_reduce_chunks<<<(unsigned)((3 * d + 255) / 256), 256, 0, ctx->stream>>>(csum, n_chunks, d, sums, t0 > 0);
    dbgz_count_launch(ctx);
    // dU[l, t] += sum_n y[l][n] (p sbar)[t][n] over the chunk's samples:
    // (d x Nc) x (Nc x d), sample-contiguous rows of leading dimension N
    if (want_U) {
      const int nc = (int)((t1 - t0) * 128);
      if (precision == DBGZ_PREC_FP64) {
        // dU[l, t] (+)= sum_n Y[n, l] SB[n, t] for l < t, Y and SB the stored
        // rows as N x d column-major matrices
        dense64::GemmArgs g;
        g.m = g.n = d;
        g.k = nc;
        g.A = (const double *)ga.y;
        g.lda = N;
        g.B = (const double *)ga.sbar;
        g.ldb = N;
        g.C = (double *)dU;
        g.ldc = d;
        g.out = dense64::kOutStrictUpper;
        g.accumulate = t0 > 0;
        // split over samples: about four CTAs per SM, at least 1024 samples each
        const int64_t nt = (d + dense64::BM - 1) / dense64::BM;
        const int64_t tiles = nt * (nt + 1) / 2;
        int64_t sp = (4 * (int64_t)ctx->num_sms + tiles - 1) / tiles;
        sp = std::max<int64_t>(1, std::min<int64_t>(sp, std::min<int64_t>(64, nc / 1024)));
        g.splits = (int)sp;
        DBGZ_TRY(dbgz_ensure(ctx, du_work, std::max<size_t>(8, dense64::gemm64_partial_bytes(g))));
        g.partial = (double *)du_work.p;
        int nl = 0;
        const cudaError_t ce = dense64::gemm64<true, false>(g, ctx->stream, &nl);
        for (int i = 0; i < nl; ++i) dbgz_count_launch(ctx);
        if (ce != cudaSuccess)
          return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_grad: FP64 factor-gradient GEMM launch failed (%s)",
                           cudaGetErrorString(ce));
      } else {
        // the strict upper triangle only, on tcgen05 (du_gemm.cu)
        DBGZ_TRY(dbgz_du_gemm_tf32(ctx, d, (const float *)ga.y, (const float *)ga.sbar, nc, (float *)dU, t0 > 0,
                                   du_work));
      }
    }
  }
  DBGZ_TRY(dbgz_finalize_pass(p, (const double *)p->partials.p, tps, 0, m, (double *)p->reps.p));
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  const double inv = 1.0 / ((double)m * (double)n_reps);
  k_grad_assemble<<<dim3(sparse ? 1u : (unsigned)((d + 255) / 256), (unsigned)d), 256, 0, ctx->stream>>>(
      dU, (int)esz, sums, (const int64_t *)p->perm.p, (const double *)p->scale.p, inv, d, dU64, da_o, db_o);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  if (dP_dSigma) DBGZ_TRY(dbgz_sigma_adjoint_dev(p, dU64, da_o, db_o, dP_dSigma));
  std::vector<double> reps(n_reps);
  int dev_status = 0;
  cudaMemcpyAsync(reps.data(), p->reps.p, 8 * n_reps, cudaMemcpyDeviceToHost, ctx->stream);
  if (dP_da) cudaMemcpyAsync(dP_da, da_o, 8 * d, cudaMemcpyDeviceToHost, ctx->stream);
  if (dP_db) cudaMemcpyAsync(dP_db, db_o, 8 * d, cudaMemcpyDeviceToHost, ctx->stream);
  if (dP_dU) cudaMemcpyAsync(dP_dU, dU64, 8 * (size_t)d * d, cudaMemcpyDeviceToHost, ctx->stream);
  if (tensor || (want_U && precision != DBGZ_PREC_FP64))
    cudaMemcpyAsync(&dev_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (prof) cudaEventRecord(ctx->ev[1], ctx->stream);
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (dev_status != 0)
    return dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm_grad: a bounded wait in a tensor-core kernel gave up");
  if (prof) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->prof.pnorm_ms = ms;
    ctx->prof.kernel_launches = ctx->launch_count - launches0;
    ctx->prof.loop_launches = 2;
  }
  double res = 0.0;
  for (double v : reps) res += v;
  res /= (double)n_reps;
  double acc = 0.0;
  for (double v : reps) acc += (v - res) * (v - res) / (double)n_reps;
  *result = res;
  *err = 3.0 * std::sqrt(acc / (double)(n_reps - 1));
  *n_pts = m;
  return DBGZ_OK;
}

extern "C" int dbgz_pnorm_grad(dbgz_problem *p, int precision, double *result, double *err, int64_t *n_pts,
                               double *dP_da, double *dP_db, double *dP_dU) {
  return grad_impl(p, precision, result, err, n_pts, dP_da, dP_db, dP_dU, nullptr);
}

extern "C" int dbgz_pnorm_grad_sigma(dbgz_problem *p, int precision, double *result, double *err, int64_t *n_pts,
                                     double *dP_da, double *dP_db, double *dP_dSigma) {
  if (!dP_dSigma) return DBGZ_ERR_INVALID_ARGUMENT;
  return grad_impl(p, precision, result, err, n_pts, dP_da, dP_db, nullptr, dP_dSigma);
}

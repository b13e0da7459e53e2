// batch.cu -- dbgz_pnorm_batch: many independent problems in a few launches.
//
// The workload is thousands of small problems (d = 16..256) with one pass
// of m points x n_reps shifts each.  One problem alone is far too small to
// fill 148 SMs (a d = 16 problem is 16 sequential steps per sample), so the
// batch is factorised and integrated in three launches over all problems:
//   1. k_prepare_batch: one CTA per problem runs the whole constructor of
//      the one-problem path -- correlation scaling, the pivoted Genz
//      Cholesky (cholk::genz_block_dev / schur_tile_dev, the same code and
//      bits as chol.cu), truncation, the per-target constants, the FP32
//      copy of U and the first dimension's CDF;
//   2. simt::k_genz_simt_batch: persistent CTAs take work items (a run of
//      tiles of one problem, about the same number of tile-dimensions per
//      item, largest problems first) from a global counter and run the SIMT
//      loop of loop_simt_kernels.cuh on them.  The SIMT loop and not the
//      tensor-core loop: at d <= 512 the contraction is a small share of the
//      per-sample work (d/2 FMAs per dimension against the step's special
//      functions), and one tcgen05 tile pipeline per problem would idle;
//   3. k_finalize_batch: per (problem, shift) sums of the tile sums in tile
//      order (the one-problem finalize, so results agree bit for bit).
// Limits: 2 <= d <= min(512, chol_block_size2) (one Cholesky panel), one
// pass (n_pts = m), erf-form CDF.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "chol_dev.cuh"
#include "detmath.h"
#include "internal.cuh"
#include "loop_simt_kernels.cuh"

namespace {

using simt::BatchItem;
using simt::SimtParams;

struct BatchProb {
  int64_t d, off2, off1, offs;  // offsets into the packed d^2, d and (d-1) n_reps arrays
};

template <typename T>
__global__ void __launch_bounds__(256) k_prepare_batch(const BatchProb *probs, double *M_all, double *a_all,
                                                       double *b_all, int64_t *perm_all, double *scale_all,
                                                       double *work_all, int64_t *rank_all, float *U32_all,
                                                       TargetParams64 *t64_all, TargetParams32 *t32_all,
                                                       SimtParams<T> *params, double *first3, int *flags,
                                                       int64_t bs1) {
  const BatchProb P = probs[blockIdx.x];
  const int64_t n = P.d;
  double *M = M_all + P.off2, *a = a_all + P.off1, *b = b_all + P.off1, *scale = scale_all + P.off1;
  int64_t *perm = perm_all + P.off1, *rank = rank_all + blockIdx.x;
  double *dvec = work_all + 3 * P.off1, *svec = dvec + n, *ovec = svec + n;
  const int tid = threadIdx.x, nt = blockDim.x;
  extern __shared__ double genz_sh[];  // the panel's vectors, cholk::genz_block_smem_bytes(n)
  __shared__ double red[32];
  __shared__ double eps0;
  __shared__ int any_nan, bad;
  // eps0 = eps * max |diag| (NaN if any diagonal is NaN), src/cholesky.jl:452-456
  if (tid == 0) any_nan = bad = 0;
  __syncthreads();
  // input checks (flags[k]: 1 = a non-finite Sigma entry, 2 = a NaN bound or
  // a > b); the factorisation still runs, on whatever the values are
  {
    int f = 0;
    for (int64_t e = tid; e < n * n; e += nt)
      if (!isfinite(M[e])) f |= 1;
    for (int64_t i = tid; i < n; i += nt)
      if (isnan(a[i]) || isnan(b[i]) || a[i] > b[i]) f |= 2;
    if (f) atomicOr(&bad, f);
    __syncthreads();
    if (tid == 0) flags[blockIdx.x] = bad;
  }
  double mx = 0.0;
  for (int64_t j = tid; j < n; j += nt) {
    const double v = fabs(M[j * n + j]);
    if (v != v) any_nan = 1;
    else if (v > mx) mx = v;
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) red[tid >> 5] = mx;
  __syncthreads();
  if (tid == 0) {
    double r = 0.0;
    for (int w = 0; w < nt / 32; ++w) r = fmax(r, red[w]);
    eps0 = any_nan ? NAN : dm_mul(DBL_EPSILON, r);
  }
  // scale vector, then the correlation scaling with the mirror copy
  for (int64_t j = tid; j < n; j += nt) {
    const double v = M[j * n + j];
    scale[j] = v > 0 ? dm_sqrt(v) : 1.0;
  }
  __syncthreads();
  for (int64_t e = tid; e < n * n; e += nt) {
    const int64_t j = e / n, i = e - j * n;
    if (i > j) continue;
    const double inv_s_j = dm_div(1.0, scale[j]);
    if (i == j) {
      M[j * n + j] = 1.0;
      a[j] = dm_mul(a[j], inv_s_j);
      b[j] = dm_mul(b[j], inv_s_j);
    } else {
      const double val = dm_mul(M[j * n + i], dm_div(inv_s_j, scale[i]));
      M[j * n + i] = val;
      M[i * n + j] = val;
    }
  }
  for (int64_t i = tid; i < n; i += nt) {
    perm[i] = i;
    dvec[i] = svec[i] = ovec[i] = 0.0;
  }
  if (tid == 0) rank[0] = n;
  __syncthreads();
  // one bs2 panel [0, n-1]: Genz blocks of bs1 and the panel's Schur updates
  for (int64_t i0 = 0; i0 < n; i0 += bs1) {
    const int64_t i1 = i0 + bs1 - 1 < n - 1 ? i0 + bs1 - 1 : n - 1;
    cholk::genz_block_smem(M, n, a, b, dvec, svec, perm, i0, i1, n - 1, &eps0, rank, genz_sh);
    __syncthreads();
    if (i1 < n - 1) {
      const int64_t c0 = i1 + 1, ntl = (n - 1 - c0 + cholk::kTile) / cholk::kTile;
      for (int64_t ty = 0; ty < ntl; ++ty)
        for (int64_t tx = 0; tx < ntl; ++tx)
          cholk::schur_tile_dev(M, n, i0, i1, c0, n - 1, 1, c0 + tx * cholk::kTile, c0 + ty * cholk::kTile);
    }
    __syncthreads();
  }
  // truncate |U_ij| < eps/(9d), src/qmc.jl:133-142
  const double min_val = DBL_EPSILON / (double)(n * 9);
  for (int64_t e = tid; e < n * n; e += nt)
    if (fabs(M[e]) < min_val) M[e] = 0.0;
  __syncthreads();
  // per-target constants and the FP32 factor
  TargetParams64 *t64 = t64_all + P.off1;
  TargetParams32 *t32 = t32_all + P.off1;
  for (int64_t t = tid; t < n; t += nt) {
    const double inv_u = 1.0 / (M[t * n + t] * sqrt(2.0));
    t64[t] = TargetParams64{a[t], b[t], inv_u};
    t32[t] = TargetParams32{(float)a[t], (float)b[t], (float)inv_u, 0.f};
  }
  float *U32 = U32_all + P.off2;
  for (int64_t e = tid; e < n * n; e += nt) U32[e] = (float)M[e];
  // the first dimension's CDF, src/qmc.jl:800-809 (erf form)
  if (tid == 0) {
    const double arg_a = a[0] / (M[0] * sqrt(2.0)), arg_b = b[0] / (M[0] * sqrt(2.0));
    const double c1 = 0.5 * (1.0 + erf(arg_a)), dc1 = 0.5 * (erf(arg_b) - erf(arg_a));
    params[blockIdx.x].c1 = c1;
    params[blockIdx.x].dc1 = dc1;
    params[blockIdx.x].up1 = 1.0 - c1 - dc1;
    first3[3 * blockIdx.x] = c1;
    first3[3 * blockIdx.x + 1] = dc1;
    first3[3 * blockIdx.x + 2] = 1.0 - c1 - dc1;
  }
}

// FP32 copies of the Richtmyer shifts; *bad = 1 if one lies outside [0, 1]
// (or is NaN).
__global__ void k_shifts32(const double *sh, int64_t n, float *s32, int *bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = sh[i];
    if (!(v >= 0.0 && v <= 1.0)) atomicOr(bad, 1);
    s32[i] = (float)v;
  }
}

// Per (problem, shift): the Neumaier sum of the shift's tile sums in tile
// order and its mean, as simt::k_finalize does for one problem.
__global__ void k_finalize_batch(const double *partials, const int64_t *part_off, int64_t tps, int64_t n_reps,
                                 int64_t n_probs, int64_t m, double *reps) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= n_probs * n_reps) return;
  const int64_t prob = g / n_reps, k = g - prob * n_reps;
  const double *pk = partials + part_off[prob] + k * tps;
  double s = 0.0, c = 0.0;
  for (int64_t t = 0; t < tps; ++t) {
    const double x = pk[t];
    const double tt = s + x;
    if (fabs(s) >= fabs(x)) c += (s - tt) + x;
    else c += (x - tt) + s;
    s = tt;
  }
  s += c;
  const double inv_tot = 1.0 / (double)m;
  reps[g] = fma(0.0, 0.0, s * inv_tot);
}

template <typename T, int GEN>
int launch_batch_loop(dbgz_ctx *ctx, const SimtParams<T> *d_params, const BatchItem *d_items, int64_t n_items,
                      unsigned long long *d_counter, T *yws, int64_t Dp, int64_t grid) {
  using Pol = pol::Forward<T, GEN, false>;
  const size_t smem = sizeof(simt::SimtSmem<T>);
  auto kern = simt::k_genz_simt_batch<T, Pol>;
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(d_counter, 0, sizeof(unsigned long long), ctx->stream));
  kern<<<(unsigned)grid, simt::NT, smem, ctx->stream>>>(d_params, d_items, n_items, d_counter, yws, Dp);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

template <typename T>
int batch_grid(dbgz_ctx *ctx, int GEN, int64_t *grid) {
  const size_t smem = sizeof(simt::SimtSmem<T>);
  int per_sm = 0;
  cudaError_t e;
  if (GEN == DBGZ_QMC_SOBOL) {
    auto k = simt::k_genz_simt_batch<T, pol::Forward<T, DBGZ_QMC_SOBOL, false>>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, simt::NT, smem);
  } else {
    auto k = simt::k_genz_simt_batch<T, pol::Forward<T, DBGZ_QMC_RICHTMYER, false>>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, simt::NT, smem);
  }
  if (e != cudaSuccess || per_sm < 1) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_batch: loop kernel does not fit");
  *grid = (int64_t)per_sm * ctx->num_sms;
  return DBGZ_OK;
}


// Default choices before (or without) dbgz_batch_autotune: the tensor-core
// loop from d = 25 in the tensor-core precisions (below that the SIMT loop
// is as fast or faster: measured on B200, 2^14 points x 8 shifts), SIMT work
// items of about 1024 tile-dimensions.
constexpr int64_t kDefaultItemDims = 1024;
constexpr int64_t kDefaultTensorMinD = 25;

bool tensor_precision(int precision) {
  return precision == DBGZ_PREC_FP32_SPLIT_BF16 || precision == DBGZ_PREC_FP32_TF32;
}

void choice_for(const dbgz_ctx *ctx, int precision, int qmc_type, int64_t d, bool *tensor, int64_t *item_dims) {
  const BatchTuning &T = ctx->batch_tune[precision & 3][qmc_type & 1];
  const bool can_tensor = tensor_precision(precision) && d - 1 <= 256;
  if (T.tuned && d >= 2 && d <= kBatchMaxD) {
    *tensor = can_tensor && T.engine[d] == 1;
    *item_dims = T.item_dims[d] > 0 ? T.item_dims[d] : kDefaultItemDims;
  } else {
    *tensor = can_tensor && d >= kDefaultTensorMinD;
    *item_dims = kDefaultItemDims;
  }
}

// Forced choices for every problem of a plan (autotuner pilots).
struct ForcedChoice {
  int engine = -1;         // -1: the context's table; 0: SIMT; 1: tensor-core loop
  int64_t item_dims = 0;  // 0: the context's table
};

}  // namespace

// A batch of problems with fixed dimensions and options: device buffers,
// tables, tensor maps and kernel configurations made once; each run uploads
// the inputs, factorises, integrates and reads back.  With `graph`, the
// per-run work is one CUDA graph reading pinned host buffers of the plan.
struct dbgz_batch_plan {
  dbgz_ctx *ctx = nullptr;
  bool fp64 = false, graph_mode = false;
  int qmc_type = 0, precision = 0, n_bits = 32;
  int64_t np = 0, R = 0, m = 0, tps = 0, Dp = 0, dmax = 0, s2 = 0, s1 = 0, ss = 0, bs1 = 64, sobol_first = 0;
  int64_t n_items = 0, grid = 0, n_tensor = 0, launches = 0;
  std::vector<int64_t> dims;
  DevBuf buf;
  double *dM = nullptr, *da = nullptr, *db = nullptr, *dscale = nullptr, *dwork = nullptr, *dsh64 = nullptr;
  double *dq = nullptr, *dpart = nullptr, *dreps = nullptr, *dfirst = nullptr;
  int64_t *dperm = nullptr, *dpo = nullptr, *drank = nullptr;
  float *dU32 = nullptr, *dsh32 = nullptr;
  TargetParams64 *dt64 = nullptr;
  TargetParams32 *dt32 = nullptr;
  void *dparams = nullptr, *dY = nullptr;
  BatchItem *ditems = nullptr;
  BatchProb *dprobs = nullptr;
  uint32_t *dV = nullptr;
  uint64_t *dush = nullptr;
  int *dflags = nullptr;  // np + 1 words: per-problem input checks, then the shift check
  unsigned long long *dcounter = nullptr;
  UmmaBatchPlan *tb = nullptr;
  // pinned host block (graph mode): inputs, then outputs
  void *hblock = nullptr;
  double *hSigma = nullptr, *ha = nullptr, *hb = nullptr, *hreps = nullptr;
  void *hsh = nullptr;
  int64_t *hrank = nullptr;
  int *hflags = nullptr, *hstatus = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

int plan_free(dbgz_batch_plan *P) {
  if (!P) return DBGZ_OK;
  if (P->ctx) cudaSetDevice(P->ctx->device);
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  if (P->ctx) cudaStreamSynchronize(P->ctx->stream);
  dbgz_umma_batch_free(P->tb);
  dbgz_release(P->buf);
  if (P->hblock) cudaFreeHost(P->hblock);
  if (P->ctx) --P->ctx->live_problems;
  delete P;
  return DBGZ_OK;
}

template <typename T>
int plan_setup(dbgz_batch_plan *P, const dbgz_opts &o, const uint32_t *dirnums, const ForcedChoice &force) {
  dbgz_ctx *ctx = P->ctx;
  const int64_t np = P->np, R = P->R, m = P->m, tps = P->tps;
  const int64_t *dims = P->dims.data();
  std::vector<BatchProb> probs(np);
  std::vector<int64_t> part_off(np);
  int64_t s2 = 0, s1 = 0, ss = 0, dmax = 0;
  for (int64_t k = 0; k < np; ++k) {
    probs[k] = BatchProb{dims[k], s2, s1, ss};
    part_off[k] = k * tps * R;
    s2 += dims[k] * dims[k];
    s1 += dims[k];
    ss += (dims[k] - 1) * R;
    dmax = std::max(dmax, dims[k]);
  }
  P->s2 = s2;
  P->s1 = s1;
  P->ss = ss;
  P->dmax = dmax;
  const int64_t Dp = ((dmax - 1 + simt::G - 1) / simt::G) * simt::G;
  P->Dp = Dp;
  // engines and work items, problems in decreasing d (longest items first)
  std::vector<int64_t> order(np);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return dims[x] > dims[y]; });
  std::vector<BatchItem> items;
  std::vector<int64_t> tensor_probs;
  for (int64_t k : order) {
    bool tensor = false;
    int64_t item_dims = kDefaultItemDims;
    choice_for(ctx, P->precision, P->qmc_type, dims[k], &tensor, &item_dims);
    if (force.engine >= 0) tensor = force.engine == 1 && tensor_precision(P->precision) && dims[k] - 1 <= 256;
    if (force.item_dims > 0) item_dims = force.item_dims;
    if (tensor) {
      tensor_probs.push_back(k);
      continue;
    }
    const int64_t nt = tps * R;
    const int64_t run = std::max<int64_t>(1, std::min<int64_t>(nt, item_dims / dims[k]));
    for (int64_t t0 = 0; t0 < nt; t0 += run)
      items.push_back(BatchItem{(int32_t)k, (int32_t)t0, (int32_t)std::min(run, nt - t0), 0});
  }
  P->n_items = (int64_t)items.size();
  P->n_tensor = (int64_t)tensor_probs.size();
  int64_t grid = 0;
  DBGZ_TRY(batch_grid<T>(ctx, P->qmc_type, &grid));
  grid = std::max<int64_t>(1, std::min<int64_t>(grid, P->n_items));
  P->grid = grid;
  // one pooled device allocation
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t szM = al(8 * (size_t)s2), sz1 = al(8 * (size_t)s1), szU32 = al(4 * (size_t)s2);
  const size_t szT64 = al(sizeof(TargetParams64) * (size_t)s1), szT32 = al(sizeof(TargetParams32) * (size_t)s1);
  const size_t szP = al(sizeof(SimtParams<T>) * (size_t)np), szI = al(sizeof(BatchItem) * std::max<size_t>(items.size(), 1));
  const size_t szS64 = al(8 * (size_t)std::max<int64_t>(ss, 1)), szS32 = al(4 * (size_t)std::max<int64_t>(ss, 1));
  const size_t szQ = al(8 * (size_t)dmax), szV = al(4 * 32 * (size_t)dmax);
  const size_t szPart = al(8 * (size_t)(np * tps * R)), szReps = al(8 * (size_t)(np * R));
  const size_t szY = al(sizeof(T) * (size_t)Dp * simt::TS * (size_t)(P->n_items ? grid : 1));
  const size_t szProbs = al(sizeof(BatchProb) * np), szPO = al(8 * (size_t)np), szRank = al(8 * (size_t)np);
  const size_t szFirst = al(3 * 8 * (size_t)np), szFlags = al(4 * (size_t)(np + 1));
  const size_t total = szM + 5 * sz1 + 3 * sz1 + szU32 + szT64 + szT32 + szP + szI + szS64 + szS32 + szQ + szV +
                       szPart + szReps + szY + szProbs + szPO + szRank + szFirst + szFlags + 512;
  DBGZ_TRY(dbgz_ensure(ctx, P->buf, total));
  char *base = (char *)P->buf.p;
  auto take = [&](size_t bytes) {
    char *r = base;
    base += bytes;
    return r;
  };
  P->dM = (double *)take(szM);
  P->da = (double *)take(sz1);
  P->db = (double *)take(sz1);
  P->dperm = (int64_t *)take(sz1);
  P->dscale = (double *)take(sz1);
  P->dwork = (double *)take(3 * sz1);
  P->dU32 = (float *)take(szU32);
  P->dt64 = (TargetParams64 *)take(szT64);
  P->dt32 = (TargetParams32 *)take(szT32);
  P->dparams = take(szP);
  P->ditems = (BatchItem *)take(szI);
  P->dsh64 = (double *)take(szS64);
  P->dsh32 = (float *)take(szS32);
  P->dq = (double *)take(szQ);
  P->dV = (uint32_t *)take(szV);
  P->dpart = (double *)take(szPart);
  P->dreps = (double *)take(szReps);
  P->dY = take(szY);
  P->dprobs = (BatchProb *)take(szProbs);
  P->dpo = (int64_t *)take(szPO);
  P->drank = (int64_t *)take(szRank);
  P->dfirst = (double *)take(szFirst);
  P->dflags = (int *)take(szFlags);
  P->dush = (uint64_t *)P->dsh64;  // Sobol shifts share the Richtmyer slot (8 bytes each)
  P->dcounter = (unsigned long long *)take(256);
  // static tables: generator constants and per-problem loop parameters
  std::vector<double> q;
  std::vector<uint32_t> V;
  if (P->qmc_type == DBGZ_QMC_RICHTMYER) {
    q.resize(std::max<int64_t>(dmax - 1, 1));
    dbgz_sqrt_primes(dmax - 1, q.data());
  } else if (!dirnums) {
    V.resize((dmax - 1) * 32);
    if (dbgz_sobol_dirnums(dmax - 1, V.data()) != DBGZ_OK)
      return dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "pnorm_batch: no Sobol table for %lld dims", (long long)(dmax - 1));
    dirnums = V.data();
  }
  std::vector<SimtParams<T>> hp(np);
  for (int64_t k = 0; k < np; ++k) {
    SimtParams<T> &S = hp[k];
    S = SimtParams<T>{};
    const BatchProb &B = probs[k];
    S.d = B.d;
    S.m = m;
    S.n_reps = R;
    S.tiles_per_shift = tps;
    S.n_tiles = tps * R;
    S.Dp = Dp;
    S.gen.qmc_type = P->qmc_type;
    S.gen.n_bits = P->n_bits;
    S.gen.gen_base = 0;
    S.gen.sobol_first = P->sobol_first;
    S.gen.sobol_staged = P->qmc_type == DBGZ_QMC_SOBOL;
    S.gen.q = P->dq;
    S.gen.shift64 = P->dsh64 + B.offs;
    S.gen.shift32 = P->dsh32 + B.offs;
    S.gen.V = P->dV;
    S.gen.ushift = P->dush + B.offs;
    S.U = sizeof(T) == 8 ? (const T *)(P->dM + B.off2) : (const T *)(P->dU32 + B.off2);
    S.tgt = sizeof(T) == 8 ? (const typename simt::TgtOf<T>::type *)(P->dt64 + B.off1)
                           : (const typename simt::TgtOf<T>::type *)(P->dt32 + B.off1);
    S.cdf_form = DBGZ_CDF_ERF;
    S.yws = (T *)P->dY;
    S.partials = P->dpart + part_off[k];
  }
  cudaStream_t st = ctx->stream;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dprobs, probs.data(), sizeof(BatchProb) * np, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dpo, part_off.data(), 8 * np, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dparams, hp.data(), sizeof(SimtParams<T>) * np, cudaMemcpyHostToDevice, st));
  if (!items.empty())
    DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->ditems, items.data(), sizeof(BatchItem) * items.size(),
                                       cudaMemcpyHostToDevice, st));
  if (P->qmc_type == DBGZ_QMC_RICHTMYER)
    DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dq, q.data(), 8 * q.size(), cudaMemcpyHostToDevice, st));
  else
    DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dV, dirnums, 4 * 32 * (size_t)(dmax - 1), cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // the prepare kernel's shared memory (attribute set outside any capture)
  const int smb = (int)cholk::genz_block_smem_bytes(dmax);
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(k_prepare_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smb));
  // the tensor-core part
  if (!tensor_probs.empty()) {
    UmmaBatchArgs A;
    A.qmc_type = P->qmc_type;
    A.n_bits = P->n_bits;
    A.m = m;
    A.n_reps = R;
    A.tiles_per_shift = tps;
    A.sobol_first = P->sobol_first;
    A.probs = tensor_probs;
    std::vector<int64_t> h_off2(np), h_off1(np), h_offs(np);
    for (int64_t k = 0; k < np; ++k) {
      h_off2[k] = probs[k].off2;
      h_off1[k] = probs[k].off1;
      h_offs[k] = probs[k].offs;
    }
    A.dims = dims;
    A.off2 = h_off2.data();
    A.off1 = h_off1.data();
    A.offs = h_offs.data();
    A.part_off = part_off.data();
    A.dM = P->dM;
    A.dfirst = P->dfirst;
    A.dq = P->dq;
    A.dU32 = P->dU32;
    A.dsh32 = P->qmc_type == DBGZ_QMC_RICHTMYER ? P->dsh32 : nullptr;
    A.dt32 = P->dt32;
    A.dV = P->qmc_type == DBGZ_QMC_SOBOL ? P->dV : nullptr;
    A.dush = P->qmc_type == DBGZ_QMC_SOBOL ? P->dush : nullptr;
    A.dpart = P->dpart;
    DBGZ_TRY(dbgz_umma_batch_setup(ctx, P->precision, A, &P->tb));
  }
  return DBGZ_OK;
}

// Records timing event i of the context on the plan's stream (an event node
// of the graph while capturing).
void plan_event(dbgz_batch_plan *P, int i, bool capturing) {
  if (!P->ctx->profiling) return;
  cudaEventRecordWithFlags(P->ctx->ev[i], P->ctx->stream, capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

// The per-run work on the context's stream: uploads from the given host
// buffers, checks, factorisation, loops, reduction, read-back into the given
// host outputs.  No allocation and no synchronisation (capturable).
template <typename T>
int plan_enqueue(dbgz_batch_plan *P, const double *Sigma, const double *a, const double *b, const void *shifts,
                 double *reps, int64_t *ranks, int *flags, int *status, bool capturing) {
  dbgz_ctx *ctx = P->ctx;
  cudaStream_t st = ctx->stream;
  const int64_t np = P->np;
  int64_t launches = 0;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dM, Sigma, 8 * (size_t)P->s2, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->da, a, 8 * (size_t)P->s1, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->db, b, 8 * (size_t)P->s1, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(P->dsh64, shifts, 8 * (size_t)P->ss, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(P->dflags + np, 0, sizeof(int), st));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  if (P->qmc_type == DBGZ_QMC_RICHTMYER) {
    k_shifts32<<<(unsigned)std::min<int64_t>((P->ss + 255) / 256, 4096), 256, 0, st>>>(P->dsh64, P->ss, P->dsh32,
                                                                                         P->dflags + np);
    ++launches;
  }
  plan_event(P, 2, capturing);
  k_prepare_batch<T><<<(unsigned)np, 256, (int)cholk::genz_block_smem_bytes(P->dmax), st>>>(
      P->dprobs, P->dM, P->da, P->db, P->dperm, P->dscale, P->dwork, P->drank, P->dU32, P->dt64, P->dt32,
      (SimtParams<T> *)P->dparams, P->dfirst, P->dflags, P->bs1);
  ++launches;
  plan_event(P, 3, capturing);
  if (P->tb) {
    DBGZ_TRY(dbgz_umma_batch_enqueue(P->tb));
    launches += 2;
  }
  if (P->n_items) {
    using PolS = pol::Forward<T, DBGZ_QMC_SOBOL, false>;
    using PolR = pol::Forward<T, DBGZ_QMC_RICHTMYER, false>;
    auto kern = P->qmc_type == DBGZ_QMC_SOBOL ? simt::k_genz_simt_batch<T, PolS> : simt::k_genz_simt_batch<T, PolR>;
    DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(P->dcounter, 0, sizeof(unsigned long long), st));
    kern<<<(unsigned)P->grid, simt::NT, sizeof(simt::SimtSmem<T>), st>>>(
        (const SimtParams<T> *)P->dparams, P->ditems, P->n_items, P->dcounter, (T *)P->dY, P->Dp);
    ++launches;
  }
  plan_event(P, 4, capturing);
  k_finalize_batch<<<(unsigned)((np * P->R + 127) / 128), 128, 0, st>>>(P->dpart, P->dpo, P->tps, P->R, np, P->m,
                                                                          P->dreps);
  ++launches;
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(reps, P->dreps, 8 * (size_t)(np * P->R), cudaMemcpyDeviceToHost, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(ranks, P->drank, 8 * (size_t)np, cudaMemcpyDeviceToHost, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(flags, P->dflags, 4 * (size_t)(np + 1), cudaMemcpyDeviceToHost, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  P->launches = launches;
  if (!capturing) dbgz_count_launch(ctx, (int)launches);
  return DBGZ_OK;
}

int enqueue_any(dbgz_batch_plan *P, const double *Sigma, const double *a, const double *b, const void *shifts,
                double *reps, int64_t *ranks, int *flags, int *status, bool capturing) {
  return P->fp64 ? plan_enqueue<double>(P, Sigma, a, b, shifts, reps, ranks, flags, status, capturing)
                 : plan_enqueue<float>(P, Sigma, a, b, shifts, reps, ranks, flags, status, capturing);
}

// Results from the read-back: P and 3 SEM per problem (the one-problem
// formulas), input and rank checks.
int plan_results(dbgz_batch_plan *P, const double *reps, const int64_t *rk, const int *flags, int status,
                 double *results, double *errs, int64_t *ranks) {
  dbgz_ctx *ctx = P->ctx;
  const int64_t np = P->np, R = P->R;
  if (status != 0) return dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm_batch: a bounded wait in the tensor-core loop gave up");
  for (int64_t k = 0; k < np; ++k) {
    if (flags[k] & 1)
      return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "pnorm_batch: non-finite Sigma in problem %lld", (long long)k);
    if (flags[k] & 2)
      return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "pnorm_batch: bad bounds (NaN or a > b) in problem %lld",
                       (long long)k);
  }
  if (flags[np]) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: shifts must lie in [0,1]");
  bool fail = false;
  for (int64_t k = 0; k < np; ++k) {
    const double *v = reps + k * R;
    double res = 0.0;
    for (int64_t i = 0; i < R; ++i) res += v[i];
    res /= (double)R;
    double acc = 0.0;
    for (int64_t i = 0; i < R; ++i) acc += (v[i] - res) * (v[i] - res) / (double)R;
    const bool full = rk[k] == P->dims[k];
    fail = fail || !full;
    results[k] = full ? res : NAN;
    if (errs) errs[k] = full ? 3.0 * std::sqrt(acc / (double)(R - 1)) : NAN;
    if (ranks) ranks[k] = rk[k];
  }
  if (fail)
    return dbgz_fail(ctx, DBGZ_ERR_RANK_DEFICIENT,
                     "pnorm_batch: some problems are not full rank (their result is NaN; see ranks)");
  return DBGZ_OK;
}

void plan_profile(dbgz_batch_plan *P) {
  dbgz_ctx *ctx = P->ctx;
  if (!ctx->profiling) return;
  dbgz_profile pr = ctx->prof;
  float ms = 0.f;
  pr.pnorm_ms = 0;
  if (cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]) == cudaSuccess) pr.pnorm_ms = ms;
  if (cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]) == cudaSuccess) pr.prepare_ms = ms;
  if (cudaEventElapsedTime(&ms, ctx->ev[3], ctx->ev[4]) == cudaSuccess) pr.loop_ms = ms;
  pr.loop_launches = (P->tb ? 1 : 0) + (P->n_items ? 1 : 0);
  pr.prepare_launches = 1;
  pr.kernel_launches = P->launches;
  ctx->prof = pr;
}

int check_batch_args(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const dbgz_opts *opts, int qmc_type,
                     int precision) {
  if (!ctx || n_problems < 1 || !dims || !opts) return DBGZ_ERR_INVALID_ARGUMENT;
  const dbgz_opts &o = *opts;
  if (o.m < 1 || o.n_reps < 2 || o.chol_block_size < 1 || o.chol_block_size2 < 1 || o.n_bits < 1 || o.n_bits > 64)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: bad options");
  if (qmc_type != DBGZ_QMC_RICHTMYER && qmc_type != DBGZ_QMC_SOBOL)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: bad generator %d", qmc_type);
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: bad precision %d", precision);
  const int64_t dlim = std::min<int64_t>(kBatchMaxD, o.chol_block_size2);
  for (int64_t k = 0; k < n_problems; ++k)
    if (dims[k] < 2 || dims[k] > dlim)
      return dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "pnorm_batch: problem %lld has d = %lld (2..%lld)", (long long)k,
                       (long long)dims[k], (long long)dlim);
  const int64_t tps = (o.m + simt::TS - 1) / simt::TS;
  if (tps * o.n_reps > INT32_MAX / 2)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: too many tiles per problem");
  return DBGZ_OK;
}

int plan_create(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const dbgz_opts *opts, int qmc_type,
                int precision, const uint32_t *sobol_dirnums, int64_t sobol_first, bool graph,
                const ForcedChoice &force, dbgz_batch_plan **out) {
  DBGZ_TRY(check_batch_args(ctx, n_problems, dims, opts, qmc_type, precision));
  cudaSetDevice(ctx->device);
  dbgz_batch_plan *P = new dbgz_batch_plan;
  P->ctx = ctx;
  ++ctx->live_problems;
  P->fp64 = precision == DBGZ_PREC_FP64;
  P->graph_mode = graph;
  P->qmc_type = qmc_type;
  P->precision = precision;
  P->n_bits = (int)opts->n_bits;
  P->np = n_problems;
  P->R = opts->n_reps;
  P->m = opts->m;
  P->tps = (opts->m + simt::TS - 1) / simt::TS;
  P->bs1 = opts->chol_block_size;
  P->sobol_first = sobol_first;
  P->dims.assign(dims, dims + n_problems);
  int rc = P->fp64 ? plan_setup<double>(P, *opts, sobol_dirnums, force)
                   : plan_setup<float>(P, *opts, sobol_dirnums, force);
  if (rc == DBGZ_OK && graph) {
    // pinned host buffers: inputs (Sigma, a, b, shifts), then outputs
    const size_t in_bytes = 8 * (size_t)(P->s2 + 2 * P->s1 + P->ss);
    const size_t out_bytes = 8 * (size_t)(P->np * P->R + P->np) + 4 * (size_t)(P->np + 2);
    if (cudaHostAlloc(&P->hblock, in_bytes + out_bytes, cudaHostAllocDefault) != cudaSuccess) {
      P->hblock = nullptr;
      rc = dbgz_fail(ctx, DBGZ_ERR_OUT_OF_MEMORY, "batch plan: pinned host allocation of %zu bytes failed",
                     in_bytes + out_bytes);
    } else {
      double *h = (double *)P->hblock;
      P->hSigma = h;
      P->ha = h + P->s2;
      P->hb = P->ha + P->s1;
      P->hsh = P->hb + P->s1;
      P->hreps = (double *)P->hsh + P->ss;
      P->hrank = (int64_t *)(P->hreps + P->np * P->R);
      P->hflags = (int *)(P->hrank + P->np);
      P->hstatus = P->hflags + P->np + 1;
      std::memset(P->hblock, 0, in_bytes + out_bytes);
      cudaStreamCaptureStatus cs;
      if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch plan: the context's stream is being captured");
      } else if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch plan: stream capture failed to start");
      } else {
        const int64_t lc = ctx->launch_count;
        const int erc = enqueue_any(P, P->hSigma, P->ha, P->hb, P->hsh, P->hreps, P->hrank, P->hflags, P->hstatus,
                                    true);
        ctx->launch_count = lc;
        const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &P->graph);
        if (erc != DBGZ_OK) rc = erc;
        else if (ce != cudaSuccess || !P->graph)
          rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch plan: stream capture failed (%s)", cudaGetErrorString(ce));
        else if (cudaGraphInstantiate(&P->exec, P->graph, 0) != cudaSuccess)
          rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch plan: graph instantiation failed");
        cudaGetLastError();
      }
    }
  }
  if (rc != DBGZ_OK) {
    plan_free(P);
    return rc;
  }
  *out = P;
  return DBGZ_OK;
}

int plan_run_graph(dbgz_batch_plan *P, double *results, double *errs, int64_t *ranks) {
  dbgz_ctx *ctx = P->ctx;
  cudaSetDevice(ctx->device);
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], ctx->stream);
  DBGZ_CUDA_TRY(ctx, cudaGraphLaunch(P->exec, ctx->stream));
  if (ctx->profiling) cudaEventRecord(ctx->ev[1], ctx->stream);
  dbgz_count_launch(ctx, (int)P->launches);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch plan: %s", cudaGetErrorString(cudaGetLastError()));
  plan_profile(P);
  return plan_results(P, P->hreps, P->hrank, P->hflags, *P->hstatus, results, errs, ranks);
}

}  // namespace

extern "C" int dbgz_batch_plan_create(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const dbgz_opts *opts,
                                      int qmc_type, int precision, const uint32_t *sobol_dirnums,
                                      int64_t sobol_first, dbgz_batch_plan **out) {
  if (!out) return DBGZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  return plan_create(ctx, n_problems, dims, opts, qmc_type, precision, sobol_dirnums, sobol_first, true,
                     ForcedChoice{}, out);
}

extern "C" int dbgz_batch_plan_buffers(dbgz_batch_plan *plan, double **Sigma, double **a, double **b,
                                       void **shifts) {
  if (!plan) return DBGZ_ERR_INVALID_ARGUMENT;
  if (Sigma) *Sigma = plan->hSigma;
  if (a) *a = plan->ha;
  if (b) *b = plan->hb;
  if (shifts) *shifts = plan->hsh;
  return DBGZ_OK;
}

extern "C" int dbgz_batch_plan_info(const dbgz_batch_plan *plan, int64_t *n_tensor_problems, int64_t *n_simt_items,
                                    int64_t *kernels_per_run, int64_t *host_bytes) {
  if (!plan) return DBGZ_ERR_INVALID_ARGUMENT;
  if (n_tensor_problems) *n_tensor_problems = plan->n_tensor;
  if (n_simt_items) *n_simt_items = plan->n_items;
  if (kernels_per_run) *kernels_per_run = plan->launches;
  if (host_bytes) *host_bytes = 8 * (plan->s2 + 2 * plan->s1 + plan->ss);
  return DBGZ_OK;
}

extern "C" int dbgz_batch_plan_run(dbgz_batch_plan *plan, double *results, double *errs, int64_t *ranks) {
  if (!plan || !results) return DBGZ_ERR_INVALID_ARGUMENT;
  return plan_run_graph(plan, results, errs, ranks);
}

extern "C" int dbgz_batch_plan_destroy(dbgz_batch_plan *plan) { return plan_free(plan); }

extern "C" int dbgz_pnorm_batch(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const double *Sigma,
                                const double *a, const double *b, const dbgz_opts *opts, int qmc_type,
                                int precision, const double *shifts, const uint64_t *ushifts,
                                const uint32_t *sobol_dirnums, int64_t sobol_first, double *results, double *errs,
                                int64_t *ranks) {
  if (!ctx || !Sigma || !a || !b || !results) return DBGZ_ERR_INVALID_ARGUMENT;
  if (qmc_type == DBGZ_QMC_RICHTMYER ? !shifts : (qmc_type == DBGZ_QMC_SOBOL ? !ushifts : false))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: missing shifts for the generator");
  dbgz_batch_plan *P = nullptr;
  DBGZ_TRY(plan_create(ctx, n_problems, dims, opts, qmc_type, precision, sobol_dirnums, sobol_first, false,
                       ForcedChoice{}, &P));
  // one pass straight from the caller's (pageable) buffers, no graph
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], ctx->stream);
  std::vector<double> reps(P->np * P->R);
  std::vector<int64_t> rk(P->np);
  std::vector<int> flags(P->np + 1);
  int status = 0;
  const void *sh = qmc_type == DBGZ_QMC_RICHTMYER ? (const void *)shifts : (const void *)ushifts;
  int rc = enqueue_any(P, Sigma, a, b, sh, reps.data(), rk.data(), flags.data(), &status, false);
  if (ctx->profiling) cudaEventRecord(ctx->ev[1], ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && rc == DBGZ_OK)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_batch: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc == DBGZ_OK) {
    plan_profile(P);
    rc = plan_results(P, reps.data(), rk.data(), flags.data(), status, results, errs, ranks);
  }
  plan_free(P);
  return rc;
}

namespace {

// Pilot inputs of the autotuner: n problems of dimension d, equicorrelated
// (rho = 0.5), bounds [-1.5, 1.5], shifts from a fixed generator.
void pilot_inputs(int64_t n, int64_t d, int64_t R, int qmc_type, std::vector<double> &S, std::vector<double> &a,
                  std::vector<double> &b, std::vector<uint64_t> &sh) {
  S.assign((size_t)(n * d * d), 0.5);
  for (int64_t k = 0; k < n; ++k)
    for (int64_t i = 0; i < d; ++i) S[(size_t)(k * d * d + i * d + i)] = 1.0;
  a.assign((size_t)(n * d), -1.5);
  b.assign((size_t)(n * d), 1.5);
  sh.resize((size_t)(n * (d - 1) * R));
  uint64_t x = 0x9E3779B97F4A7C15ull;
  for (auto &v : sh) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    if (qmc_type == DBGZ_QMC_RICHTMYER) {
      const double u = (double)(x >> 11) * 0x1.0p-53;
      std::memcpy(&v, &u, 8);
    } else {
      v = x;
    }
  }
}

// Loop time (ms, best of `reps` runs after one warm-up) of one forced choice.
int pilot_time(dbgz_ctx *ctx, int64_t n, int64_t d, const dbgz_opts &o, int qmc_type, int precision,
               const ForcedChoice &f, const std::vector<double> &S, const std::vector<double> &a,
               const std::vector<double> &b, const std::vector<uint64_t> &sh, int reps, double *best_ms) {
  std::vector<int64_t> dims((size_t)n, d);
  dbgz_batch_plan *P = nullptr;
  DBGZ_TRY(plan_create(ctx, n, dims.data(), &o, qmc_type, precision, nullptr, 2 * o.m, false, f, &P));
  std::vector<double> rp(P->np * P->R);
  std::vector<int64_t> rk(P->np);
  std::vector<int> flags(P->np + 1);
  int status = 0, rc = DBGZ_OK;
  double best = 1e30;
  for (int it = 0; it <= reps && rc == DBGZ_OK; ++it) {
    rc = enqueue_any(P, S.data(), a.data(), b.data(), sh.data(), rp.data(), rk.data(), flags.data(), &status, false);
    if (rc == DBGZ_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "batch autotune: %s", cudaGetErrorString(cudaGetLastError()));
    if (rc == DBGZ_OK && status != 0) rc = dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "batch autotune: loop wait gave up");
    float ms = 0.f;
    if (rc == DBGZ_OK && it > 0 && cudaEventElapsedTime(&ms, ctx->ev[3], ctx->ev[4]) == cudaSuccess)
      best = std::min(best, (double)ms);
  }
  plan_free(P);
  *best_ms = best;
  return rc;
}

}  // namespace

extern "C" int dbgz_batch_autotune(dbgz_ctx *ctx, int precision, int qmc_type, const dbgz_opts *opts,
                                   int32_t *engine_out, int32_t *item_dims_out) {
  if (!ctx || !opts) return DBGZ_ERR_INVALID_ARGUMENT;
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT ||
      (qmc_type != DBGZ_QMC_RICHTMYER && qmc_type != DBGZ_QMC_SOBOL))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "batch autotune: bad precision or generator");
  dbgz_opts o = *opts;
  o.chol_block_size2 = std::max<int64_t>(o.chol_block_size2, kBatchMaxD);
  if (o.m < 1 || o.n_reps < 2) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "batch autotune: bad options");
  cudaSetDevice(ctx->device);
  // dimension buckets; each is timed at its middle dimension
  static const int64_t lo[] = {2, 17, 25, 33, 49, 65, 97, 129, 193, 258, 385};
  static const int64_t hi[] = {16, 24, 32, 48, 64, 96, 128, 192, 257, 384, 512};
  static const int64_t items[] = {256, 1024, 4096};
  const bool prof = ctx->profiling;
  ctx->profiling = true;
  BatchTuning T;
  int rc = DBGZ_OK;
  const int64_t tiles_per_prob = ((o.m + simt::TS - 1) / simt::TS) * o.n_reps;
  const int64_t target_tiles = 32 * (int64_t)ctx->num_sms;
  for (int bk = 0; bk < 11 && rc == DBGZ_OK; ++bk) {
    const int64_t d = (lo[bk] + hi[bk] + 1) / 2;
    // at least 64 problems: a batch switches problems (descriptors, tables)
    // every few tiles, and the pilot should too
    const int64_t n = std::max<int64_t>(64, (target_tiles + tiles_per_prob - 1) / tiles_per_prob);
    std::vector<double> S, a, b;
    std::vector<uint64_t> sh;
    pilot_inputs(n, d, o.n_reps, qmc_type, S, a, b, sh);
    // a choice replaces the default only when it is at least kMargin faster
    // on the pilot: the pilot stands in for the caller's problems, and a few
    // percent are within the difference between the two
    const double kMargin = 0.97;
    double best_simt = 1e30, t_def = 1e30, t = 0.0;
    int64_t best_items = kDefaultItemDims;
    for (int64_t it : items) {
      ForcedChoice f;
      f.engine = 0;
      f.item_dims = it;
      if ((rc = pilot_time(ctx, n, d, o, qmc_type, precision, f, S, a, b, sh, 2, &t))) break;
      if (it == kDefaultItemDims) t_def = t;
      if (t < best_simt) {
        best_simt = t;
        best_items = it;
      }
    }
    if (rc) break;
    if (best_simt > kMargin * t_def) {
      best_simt = t_def;
      best_items = kDefaultItemDims;
    }
    int engine = 0;
    if (tensor_precision(precision) && d - 1 <= 256) {
      ForcedChoice f;
      f.engine = 1;
      if ((rc = pilot_time(ctx, n, d, o, qmc_type, precision, f, S, a, b, sh, 2, &t))) break;
      const bool def_tensor = d >= kDefaultTensorMinD;
      engine = def_tensor ? (best_simt < kMargin * t ? 0 : 1) : (t < kMargin * best_simt ? 1 : 0);
    }
    for (int64_t dd = lo[bk]; dd <= hi[bk]; ++dd) {
      T.engine[dd] = (int8_t)(engine && dd - 1 <= 256);
      T.item_dims[dd] = (int32_t)best_items;
    }
  }
  ctx->profiling = prof;
  if (rc != DBGZ_OK) return rc;
  T.tuned = true;
  ctx->batch_tune[precision][qmc_type] = T;
  for (int64_t dd = 0; dd <= kBatchMaxD; ++dd) {
    if (engine_out) engine_out[dd] = T.engine[dd];
    if (item_dims_out) item_dims_out[dd] = T.item_dims[dd];
  }
  return DBGZ_OK;
}

extern "C" int dbgz_batch_tuning(const dbgz_ctx *ctx, int precision, int qmc_type, int32_t *engine_out,
                                 int32_t *item_dims_out, int *tuned) {
  if (!ctx || precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT ||
      (qmc_type != DBGZ_QMC_RICHTMYER && qmc_type != DBGZ_QMC_SOBOL))
    return DBGZ_ERR_INVALID_ARGUMENT;
  const BatchTuning &T = ctx->batch_tune[precision][qmc_type];
  if (tuned) *tuned = T.tuned ? 1 : 0;
  for (int64_t d = 0; d <= kBatchMaxD; ++d) {
    bool tensor = false;
    int64_t item_dims = kDefaultItemDims;
    if (d >= 2) choice_for(ctx, precision, qmc_type, d, &tensor, &item_dims);
    if (engine_out) engine_out[d] = tensor ? 1 : 0;
    if (item_dims_out) item_dims_out[d] = (int32_t)item_dims;
  }
  return DBGZ_OK;
}

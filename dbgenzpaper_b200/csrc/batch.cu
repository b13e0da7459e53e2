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
                                                       SimtParams<T> *params, double *first3, int64_t bs1) {
  const BatchProb P = probs[blockIdx.x];
  const int64_t n = P.d;
  double *M = M_all + P.off2, *a = a_all + P.off1, *b = b_all + P.off1, *scale = scale_all + P.off1;
  int64_t *perm = perm_all + P.off1, *rank = rank_all + blockIdx.x;
  double *dvec = work_all + 3 * P.off1, *svec = dvec + n, *ovec = svec + n;
  const int tid = threadIdx.x, nt = blockDim.x;
  extern __shared__ double genz_sh[];  // the panel's vectors, cholk::genz_block_smem_bytes(n)
  __shared__ double red[32];
  __shared__ double eps0;
  __shared__ int any_nan;
  // eps0 = eps * max |diag| (NaN if any diagonal is NaN), src/cholesky.jl:452-456
  if (tid == 0) any_nan = 0;
  __syncthreads();
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

// Work items: runs of tiles of about kItemDims tile-dimensions, problems in
// decreasing d (the longest items first, for the balance of the tail).
constexpr int64_t kItemDims = 1024;

template <typename T>
int run_batch(dbgz_ctx *ctx, int64_t np, const int64_t *dims, const double *Sigma, const double *a, const double *b,
              const dbgz_opts &o, int qmc_type, const double *shifts, const uint64_t *ushifts,
              const uint32_t *dirnums, int64_t sobol_first, double *results, double *errs, int64_t *ranks,
              int *any_rank_fail, int precision) {
  // tensor-core loop for the single-phase problems when a tensor-core mode is
  // asked for (FP32 only); the SIMT loop for everything else
  const bool tensor = sizeof(T) == 4 && (precision == DBGZ_PREC_FP32_SPLIT_BF16 || precision == DBGZ_PREC_FP32_TF32);
  const int64_t R = o.n_reps, m = o.m;
  const int64_t tps = (m + simt::TS - 1) / simt::TS;
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
  const int64_t Dp = ((dmax - 1 + simt::G - 1) / simt::G) * simt::G;
  // work items
  std::vector<int64_t> order(np);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return dims[x] > dims[y]; });
  std::vector<BatchItem> items;
  std::vector<int64_t> tensor_probs;
  for (int64_t k : order) {
    if (tensor && dims[k] - 1 <= 256) {
      tensor_probs.push_back(k);
      continue;
    }
    const int64_t nt = tps * R;
    const int64_t run = std::max<int64_t>(1, std::min<int64_t>(nt, kItemDims / dims[k]));
    for (int64_t t0 = 0; t0 < nt; t0 += run)
      items.push_back(BatchItem{(int32_t)k, (int32_t)t0, (int32_t)std::min(run, nt - t0), 0});
  }
  int64_t grid = 0;
  DBGZ_TRY(batch_grid<T>(ctx, qmc_type, &grid));
  grid = std::max<int64_t>(1, std::min<int64_t>(grid, (int64_t)items.size()));
  // one pooled allocation for everything
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t szM = al(8 * (size_t)s2), sz1 = al(8 * (size_t)s1), szU32 = al(4 * (size_t)s2);
  const size_t szT64 = al(sizeof(TargetParams64) * (size_t)s1), szT32 = al(sizeof(TargetParams32) * (size_t)s1);
  const size_t szP = al(sizeof(SimtParams<T>) * (size_t)np), szI = al(sizeof(BatchItem) * items.size());
  const size_t szS64 = al(8 * (size_t)std::max<int64_t>(ss, 1)), szS32 = al(4 * (size_t)std::max<int64_t>(ss, 1));
  const size_t szQ = al(8 * (size_t)dmax), szV = al(4 * 32 * (size_t)dmax);
  const size_t szPart = al(8 * (size_t)(np * tps * R)), szReps = al(8 * (size_t)(np * R));
  const size_t szY = al(sizeof(T) * (size_t)Dp * simt::TS * (size_t)grid);
  const size_t szProbs = al(sizeof(BatchProb) * np), szPO = al(8 * (size_t)np), szRank = al(8 * (size_t)np);
  const size_t szFirst = al(3 * 8 * (size_t)np);
  const size_t total = szM + 5 * sz1 + 3 * sz1 + szU32 + szT64 + szT32 + szP + szI + szS64 + szS32 + szQ + szV +
                       szPart + szReps + szY + szProbs + szPO + szRank + szFirst + 512;
  DevBuf buf;
  DBGZ_TRY(dbgz_ensure(ctx, buf, total));
  char *base = (char *)buf.p;
  auto take = [&](size_t bytes) {
    char *r = base;
    base += bytes;
    return r;
  };
  double *dM = (double *)take(szM), *da = (double *)take(sz1), *db = (double *)take(sz1);
  int64_t *dperm = (int64_t *)take(sz1);
  double *dscale = (double *)take(sz1), *dwork = (double *)take(3 * sz1);
  float *dU32 = (float *)take(szU32);
  TargetParams64 *dt64 = (TargetParams64 *)take(szT64);
  TargetParams32 *dt32 = (TargetParams32 *)take(szT32);
  SimtParams<T> *dparams = (SimtParams<T> *)take(szP);
  BatchItem *ditems = (BatchItem *)take(szI);
  double *dsh64 = (double *)take(szS64);
  float *dsh32 = (float *)take(szS32);
  double *dq = (double *)take(szQ);
  uint32_t *dV = (uint32_t *)take(szV);
  double *dpart = (double *)take(szPart), *dreps = (double *)take(szReps);
  T *dY = (T *)take(szY);
  BatchProb *dprobs = (BatchProb *)take(szProbs);
  int64_t *dpo = (int64_t *)take(szPO), *drank = (int64_t *)take(szRank);
  double *dfirst = (double *)take(szFirst);
  uint64_t *dush = (uint64_t *)dsh64;  // Sobol shifts share the Richtmyer slot (8 bytes each)
  unsigned long long *dcounter = (unsigned long long *)take(256);
  cudaStream_t st = ctx->stream;
  int rc = DBGZ_OK;
  do {
    // host-side tables: generator constants and per-problem loop parameters
    std::vector<double> q;
    std::vector<uint32_t> V;
    std::vector<float> s32;
    if (qmc_type == DBGZ_QMC_RICHTMYER) {
      q.resize(std::max<int64_t>(dmax - 1, 1));
      dbgz_sqrt_primes(dmax - 1, q.data());
      s32.resize(ss);
      for (int64_t i = 0; i < ss; ++i) s32[i] = (float)shifts[i];
    } else if (!dirnums) {
      V.resize((dmax - 1) * 32);
      if (dbgz_sobol_dirnums(dmax - 1, V.data()) != DBGZ_OK) {
        rc = dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "pnorm_batch: no Sobol table for %lld dims", (long long)(dmax - 1));
        break;
      }
      dirnums = V.data();
    }
    std::vector<SimtParams<T>> hp(np);
    for (int64_t k = 0; k < np; ++k) {
      SimtParams<T> &P = hp[k];
      P = SimtParams<T>{};
      const BatchProb &B = probs[k];
      P.d = B.d;
      P.m = m;
      P.n_reps = R;
      P.tiles_per_shift = tps;
      P.n_tiles = tps * R;
      P.Dp = Dp;
      P.gen.qmc_type = qmc_type;
      P.gen.n_bits = (int)o.n_bits;
      P.gen.gen_base = 0;
      P.gen.sobol_first = sobol_first;
      P.gen.q = dq;
      P.gen.shift64 = dsh64 + B.offs;
      P.gen.shift32 = dsh32 + B.offs;
      P.gen.V = dV;
      P.gen.ushift = dush + B.offs;
      P.U = sizeof(T) == 8 ? (const T *)(dM + B.off2) : (const T *)(dU32 + B.off2);
      P.tgt = sizeof(T) == 8 ? (const typename simt::TgtOf<T>::type *)(dt64 + B.off1)
                             : (const typename simt::TgtOf<T>::type *)(dt32 + B.off1);
      P.cdf_form = DBGZ_CDF_ERF;
      P.yws = dY;
      P.partials = dpart + part_off[k];
    }
    // uploads (pageable host memory: each copy is staged by the driver)
    bool ok = cudaMemcpyAsync(dM, Sigma, 8 * (size_t)s2, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(da, a, 8 * (size_t)s1, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(db, b, 8 * (size_t)s1, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dprobs, probs.data(), sizeof(BatchProb) * np, cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(dpo, part_off.data(), 8 * np, cudaMemcpyHostToDevice, st) == cudaSuccess &&
              cudaMemcpyAsync(dparams, hp.data(), sizeof(SimtParams<T>) * np, cudaMemcpyHostToDevice, st) ==
                  cudaSuccess &&
              cudaMemcpyAsync(ditems, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice,
                              st) == cudaSuccess;
    if (ok && qmc_type == DBGZ_QMC_RICHTMYER)
      ok = cudaMemcpyAsync(dq, q.data(), 8 * q.size(), cudaMemcpyHostToDevice, st) == cudaSuccess &&
           cudaMemcpyAsync(dsh64, shifts, 8 * (size_t)ss, cudaMemcpyHostToDevice, st) == cudaSuccess &&
           cudaMemcpyAsync(dsh32, s32.data(), 4 * (size_t)ss, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (ok && qmc_type == DBGZ_QMC_SOBOL)
      ok = cudaMemcpyAsync(dV, dirnums, 4 * 32 * (size_t)(dmax - 1), cudaMemcpyHostToDevice, st) == cudaSuccess &&
           cudaMemcpyAsync(dush, ushifts, 8 * (size_t)ss, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (!ok) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_batch: upload failed");
      break;
    }
    if (ctx->profiling) cudaEventRecord(ctx->ev[2], st);
    {
      const int smb = (int)cholk::genz_block_smem_bytes(dmax);
      cudaFuncSetAttribute(k_prepare_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smb);
      k_prepare_batch<T><<<(unsigned)np, 256, smb, st>>>(dprobs, dM, da, db, dperm, dscale, dwork, drank, dU32,
                                                         dt64, dt32, dparams, dfirst, o.chol_block_size);
    }
    dbgz_count_launch(ctx);
    if (ctx->profiling) cudaEventRecord(ctx->ev[3], st);
    if (!tensor_probs.empty()) {
      UmmaBatchArgs A;
      A.qmc_type = qmc_type;
      A.n_bits = (int)o.n_bits;
      A.m = m;
      A.n_reps = R;
      A.tiles_per_shift = tps;
      A.sobol_first = sobol_first;
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
      A.dM = dM;
      A.dfirst = dfirst;
      A.dq = dq;
      A.dU32 = dU32;
      A.dsh32 = qmc_type == DBGZ_QMC_RICHTMYER ? dsh32 : nullptr;
      A.dt32 = dt32;
      A.dV = qmc_type == DBGZ_QMC_SOBOL ? dV : nullptr;
      A.dush = qmc_type == DBGZ_QMC_SOBOL ? dush : nullptr;
      A.dpart = dpart;
      if ((rc = dbgz_loop_umma_batch(ctx, precision, A))) break;
    }
    if (!items.empty()) {
      if (qmc_type == DBGZ_QMC_SOBOL)
        rc = launch_batch_loop<T, DBGZ_QMC_SOBOL>(ctx, dparams, ditems, (int64_t)items.size(), dcounter, dY, Dp,
                                                  grid);
      else
        rc = launch_batch_loop<T, DBGZ_QMC_RICHTMYER>(ctx, dparams, ditems, (int64_t)items.size(), dcounter, dY, Dp,
                                                      grid);
    }
    if (rc) break;
    if (ctx->profiling) cudaEventRecord(ctx->ev[4], st);
    k_finalize_batch<<<(unsigned)((np * R + 127) / 128), 128, 0, st>>>(dpart, dpo, tps, R, np, m, dreps);
    dbgz_count_launch(ctx);
    std::vector<double> reps(np * R);
    std::vector<int64_t> rk(np);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(reps.data(), dreps, 8 * reps.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(rk.data(), drank, 8 * np, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_batch: launch or copy failed");
      break;
    }
    if (ctx->profiling) cudaEventRecord(ctx->ev[1], st);
    int dev_status = 0;
    if (!tensor_probs.empty()) cudaMemcpyAsync(&dev_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_batch: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    if (dev_status != 0) {
      rc = dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm_batch: a bounded wait in the tensor-core loop gave up");
      break;
    }
    for (int64_t k = 0; k < np; ++k) {
      const double *v = reps.data() + k * R;
      double res = 0.0;
      for (int64_t i = 0; i < R; ++i) res += v[i];
      res /= (double)R;
      double acc = 0.0;
      for (int64_t i = 0; i < R; ++i) acc += (v[i] - res) * (v[i] - res) / (double)R;
      const bool full = rk[k] == dims[k];
      if (!full) *any_rank_fail = 1;
      results[k] = full ? res : NAN;
      if (errs) errs[k] = full ? 3.0 * std::sqrt(acc / (double)(R - 1)) : NAN;
      if (ranks) ranks[k] = rk[k];
    }
    if (ctx->profiling) {
      dbgz_profile pr = ctx->prof;
      pr.pnorm_ms = 0;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]) == cudaSuccess) pr.pnorm_ms = ms;
      if (cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]) == cudaSuccess) pr.prepare_ms = ms;
      if (cudaEventElapsedTime(&ms, ctx->ev[3], ctx->ev[4]) == cudaSuccess) pr.loop_ms = ms;
      pr.loop_launches = 1;
      pr.prepare_launches = 1;
      ctx->prof = pr;
    }
  } while (0);
  dbgz_release(buf);
  return rc;
}

}  // namespace

extern "C" int dbgz_pnorm_batch(dbgz_ctx *ctx, int64_t n_problems, const int64_t *dims, const double *Sigma,
                                const double *a, const double *b, const dbgz_opts *opts, int qmc_type,
                                int precision, const double *shifts, const uint64_t *ushifts,
                                const uint32_t *sobol_dirnums, int64_t sobol_first, double *results, double *errs,
                                int64_t *ranks) {
  if (!ctx || n_problems < 1 || !dims || !Sigma || !a || !b || !opts || !results)
    return DBGZ_ERR_INVALID_ARGUMENT;
  const dbgz_opts &o = *opts;
  if (o.m < 1 || o.n_reps < 2 || o.chol_block_size < 1 || o.chol_block_size2 < 1 || o.n_bits < 1 || o.n_bits > 64)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: bad options");
  if (qmc_type == DBGZ_QMC_RICHTMYER ? !shifts : (qmc_type == DBGZ_QMC_SOBOL ? !ushifts : true))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: missing shifts for the generator");
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: bad precision %d", precision);
  const int64_t dlim = std::min<int64_t>(512, o.chol_block_size2);
  int64_t s2 = 0, s1 = 0, ss = 0;
  for (int64_t k = 0; k < n_problems; ++k) {
    if (dims[k] < 2 || dims[k] > dlim)
      return dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "pnorm_batch: problem %lld has d = %lld (2..%lld)",
                       (long long)k, (long long)dims[k], (long long)dlim);
    s2 += dims[k] * dims[k];
    s1 += dims[k];
    ss += (dims[k] - 1) * o.n_reps;
  }
  for (int64_t i = 0; i < s2; ++i)
    if (!std::isfinite(Sigma[i])) return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "pnorm_batch: non-finite Sigma");
  for (int64_t i = 0; i < s1; ++i)
    if (std::isnan(a[i]) || std::isnan(b[i]) || a[i] > b[i])
      return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "pnorm_batch: bad bounds at packed index %lld", (long long)i);
  if (qmc_type == DBGZ_QMC_RICHTMYER)
    for (int64_t i = 0; i < ss; ++i)
      if (!(shifts[i] >= 0.0 && shifts[i] <= 1.0))
        return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_batch: shifts must lie in [0,1]");
  cudaSetDevice(ctx->device);
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], ctx->stream);
  int fail = 0, rc;
  if (precision == DBGZ_PREC_FP64)
    rc = run_batch<double>(ctx, n_problems, dims, Sigma, a, b, o, qmc_type, shifts, ushifts, sobol_dirnums,
                           sobol_first, results, errs, ranks, &fail, precision);
  else
    rc = run_batch<float>(ctx, n_problems, dims, Sigma, a, b, o, qmc_type, shifts, ushifts, sobol_dirnums,
                          sobol_first, results, errs, ranks, &fail, precision);
  if (rc == DBGZ_OK && fail)
    return dbgz_fail(ctx, DBGZ_ERR_RANK_DEFICIENT,
                     "pnorm_batch: some problems are not full rank (their result is NaN; see ranks)");
  return rc;
}

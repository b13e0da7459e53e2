// api.cu -- the C ABI of libdbgenz (include/dbgenz.h).
#include "internal.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

// ---------------------------------------------------------------------------
int dbgz_fail(dbgz_ctx *ctx, int status, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return status;
}

// Frees every cached block of the context's pool (cudaFree synchronises the
// device, so the blocks are idle afterwards).
static size_t pool_trim(dbgz_ctx *ctx) {
  size_t freed = 0;
  for (auto &kv : ctx->pool) {
    cudaFree(kv.second);
    freed += kv.first;
  }
  ctx->pool.clear();
  ctx->pool_bytes = 0;
  return freed;
}

int dbgz_ensure(dbgz_ctx *ctx, DevBuf &b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.p && b.bytes >= bytes) return DBGZ_OK;
  dbgz_release(b);
  // capacity classes: 512 B steps below 1 MiB, 2 MiB steps above
  const size_t want = bytes < (1u << 20) ? (bytes + 511) & ~size_t(511) : (bytes + (2u << 20) - 1) & ~size_t((2u << 20) - 1);
  // smallest cached block that fits and wastes at most a quarter (+2 MiB)
  auto it = ctx->pool.lower_bound(want);
  if (it != ctx->pool.end() && it->first <= want + want / 4 + (2u << 20)) {
    b.p = it->second;
    b.bytes = it->first;
    b.owner = ctx;
    ctx->pool_bytes -= it->first;
    ctx->pool.erase(it);
    return DBGZ_OK;
  }
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e == cudaErrorMemoryAllocation && !ctx->pool.empty()) {
    cudaGetLastError();
    pool_trim(ctx);
    e = cudaMalloc(&b.p, want);
  }
  if (e != cudaSuccess) {
    b.p = nullptr;
    cudaGetLastError();
    return dbgz_fail(ctx, e == cudaErrorMemoryAllocation ? DBGZ_ERR_OUT_OF_MEMORY : DBGZ_ERR_CUDA,
                     "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  b.bytes = want;
  b.owner = ctx;
  return DBGZ_OK;
}

void dbgz_release(DevBuf &b) {
  if (b.p) {
    if (b.owner) {
      b.owner->pool.emplace(b.bytes, b.p);
      b.owner->pool_bytes += b.bytes;
    } else {
      cudaFree(b.p);
    }
  }
  b.p = nullptr;
  b.bytes = 0;
  b.owner = nullptr;
}

// Smallest index of a non-finite entry of x[0..n) into *first (which starts
// at INT64_MAX); the prepare's check of Sigma on the device.
__global__ void k_first_nonfinite(const double *x, int64_t n, unsigned long long *first) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (!isfinite(x[i])) atomicMin(first, (unsigned long long)i);
}

static int upload(dbgz_ctx *ctx, DevBuf &b, const void *src, size_t bytes) {
  DBGZ_TRY(dbgz_ensure(ctx, b, bytes));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return DBGZ_OK;
}

// ---------------------------------------------------------------------------
extern "C" {

int dbgz_abi_version(void) { return DBGZ_ABI_VERSION; }

void dbgz_default_opts(dbgz_opts *o) {
  if (!o) return;
  o->chol_block_size = 64;
  o->chol_block_size2 = 512;
  o->m = 10000;
  o->block_size_i = 64;
  o->block_size_i2 = 32;
  o->block_size_j = 64;
  o->n_blocks = 1;
  o->n_reps = 12;
  o->n_bits = 32;
  o->max_pts = 10000;
  o->max_abs_err = 1e-6;
}

const char *dbgz_status_string(int s) {
  switch (s) {
    case DBGZ_OK: return "ok";
    case DBGZ_ERR_INVALID_ARGUMENT: return "invalid argument";
    case DBGZ_ERR_RANK_DEFICIENT: return "QMCData requires a full-rank Cholesky factorization.";
    case DBGZ_ERR_NONFINITE_INPUT: return "non-finite input";
    case DBGZ_ERR_DIMENSION: return "unsupported dimension";
    case DBGZ_ERR_OUT_OF_MEMORY: return "out of device memory";
    case DBGZ_ERR_CUDA: return "CUDA error";
    case DBGZ_ERR_TIMEOUT: return "device-side wait timed out";
    case DBGZ_ERR_UNSUPPORTED: return "unsupported mode";
    default: return "unknown status";
  }
}

int dbgz_create(int device, dbgz_ctx **out) {
  if (!out) return DBGZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return DBGZ_ERR_CUDA;
  }
  if (device < 0 || device >= n) return DBGZ_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return DBGZ_ERR_CUDA;
  dbgz_ctx *ctx = new (std::nothrow) dbgz_ctx();
  if (!ctx) return DBGZ_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&ctx->d_status, sizeof(int) * 4) != cudaSuccess) {
    delete ctx;
    return DBGZ_ERR_CUDA;
  }
  cudaMemset(ctx->d_status, 0, sizeof(int) * 4);
  for (cudaEvent_t &e : ctx->ev) cudaEventCreate(&e);
  *out = ctx;
  return DBGZ_OK;
}

int dbgz_destroy(dbgz_ctx *ctx) {
  if (!ctx) return DBGZ_ERR_INVALID_ARGUMENT;
  // problems run on the context's stream and return their buffers to its
  // pool: they must be freed first
  if (ctx->live_problems > 0)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "destroy: %lld problem(s) of this context are still alive",
                     (long long)ctx->live_problems);
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  pool_trim(ctx);
  if (ctx->d_status) cudaFree(ctx->d_status);
  for (cudaEvent_t &e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DBGZ_OK;
}

int dbgz_set_state_budget(dbgz_ctx *ctx, uint64_t bytes) {
  if (!ctx || bytes == 0) return DBGZ_ERR_INVALID_ARGUMENT;
  ctx->state_budget = (size_t)bytes;
  return DBGZ_OK;
}

int dbgz_set_grad_checkpoints(dbgz_ctx *ctx, int64_t segment) {
  if (!ctx || segment < 0) return DBGZ_ERR_INVALID_ARGUMENT;
  ctx->grad_ckpt_seg = segment;
  return DBGZ_OK;
}

int dbgz_release_cached(dbgz_ctx *ctx, uint64_t *freed_bytes) {
  if (!ctx) return DBGZ_ERR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  const size_t f = pool_trim(ctx);
  if (freed_bytes) *freed_bytes = f;
  return DBGZ_OK;
}

const char *dbgz_last_error(const dbgz_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int dbgz_set_profiling(dbgz_ctx *ctx, int enable) {
  if (!ctx) return DBGZ_ERR_INVALID_ARGUMENT;
  ctx->profiling = enable != 0;
  return DBGZ_OK;
}

int dbgz_get_profile(const dbgz_ctx *ctx, dbgz_profile *out) {
  if (!ctx || !out) return DBGZ_ERR_INVALID_ARGUMENT;
  *out = ctx->prof;
  return DBGZ_OK;
}

static float event_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  return ms;
}

// ---- primitives --------------------------------------------------------------
int dbgz_cholesky_genz(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b, int64_t bs1,
                       int64_t bs2, int64_t bs3, int64_t bs4, int64_t *perm, double *scale_vec,
                       int64_t *rank) {
  if (!ctx || !M || !a || !b || !perm || !scale_vec || !rank || d < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "cholesky_genz: bad argument");
  cudaSetDevice(ctx->device);
  DevBuf dM, da, db, dp, ds;
  int rc = DBGZ_OK;
  size_t nn = (size_t)d * d;
  if ((rc = upload(ctx, dM, M, nn * 8)) || (rc = upload(ctx, da, a, d * 8)) ||
      (rc = upload(ctx, db, b, d * 8)) || (rc = dbgz_ensure(ctx, dp, d * 8)) ||
      (rc = dbgz_ensure(ctx, ds, d * 8)))
    goto done;
  rc = dbgz_chol_genz_dev(ctx, d, (double *)dM.p, (double *)da.p, (double *)db.p, bs1, bs2, bs3,
                          bs4, (int64_t *)dp.p, (double *)ds.p, rank);
  if (rc) goto done;
  cudaMemcpyAsync(M, dM.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(a, da.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(b, db.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(perm, dp.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(scale_vec, ds.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_genz: copy back failed");
done:
  dbgz_release(dM); dbgz_release(da); dbgz_release(db); dbgz_release(dp); dbgz_release(ds);
  return rc;
}

int dbgz_cholesky_classic(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b, int64_t bs1,
                          int64_t bs2, int64_t bs3, int64_t bs4, double *scale_vec) {
  if (!ctx || !M || !a || !b || !scale_vec || d < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "cholesky_classic: bad argument");
  cudaSetDevice(ctx->device);
  DevBuf dM, da, db, ds;
  int rc = DBGZ_OK;
  size_t nn = (size_t)d * d;
  if ((rc = upload(ctx, dM, M, nn * 8)) || (rc = upload(ctx, da, a, d * 8)) ||
      (rc = upload(ctx, db, b, d * 8)) || (rc = dbgz_ensure(ctx, ds, d * 8)))
    goto done;
  rc = dbgz_chol_classic_dev(ctx, d, (double *)dM.p, (double *)da.p, (double *)db.p, bs1, bs2,
                             bs3, bs4, (double *)ds.p);
  if (rc) goto done;
  cudaMemcpyAsync(M, dM.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(a, da.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(b, db.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(scale_vec, ds.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_classic: copy back failed");
done:
  dbgz_release(dM); dbgz_release(da); dbgz_release(db); dbgz_release(ds);
  return rc;
}

int dbgz_richtmyer_mat(dbgz_ctx *ctx, int64_t m, int64_t n, const double *q, int64_t n0,
                       double *X) {
  if (!ctx || m < 0 || n < 0 || ((m * n) > 0 && (!q || !X)))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "richtmyer_mat: bad argument");
  if (m * n == 0) return DBGZ_OK;
  cudaSetDevice(ctx->device);
  DevBuf dq, dX;
  int rc = upload(ctx, dq, q, n * 8);
  if (!rc) rc = dbgz_ensure(ctx, dX, (size_t)m * n * 8);
  if (!rc) rc = dbgz_richtmyer_dev(ctx, m, n, (const double *)dq.p, n0, (double *)dX.p);
  if (!rc) {
    cudaMemcpyAsync(X, dX.p, (size_t)m * n * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "richtmyer_mat: copy back failed");
  }
  dbgz_release(dq); dbgz_release(dX);
  return rc;
}

int dbgz_sobol_mat(dbgz_ctx *ctx, int64_t m, int64_t dims, const uint32_t *V, int64_t first,
                   uint32_t *X) {
  if (!ctx || m < 0 || dims < 0 || first < 0 || ((m * dims) > 0 && (!V || !X)))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "sobol_mat: bad argument");
  if (first + m > (int64_t)1 << 32)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "sobol_mat: index beyond 2^32");
  if (m * dims == 0) return DBGZ_OK;
  cudaSetDevice(ctx->device);
  DevBuf dV, dX;
  int rc = upload(ctx, dV, V, (size_t)dims * 32 * 4);
  if (!rc) rc = dbgz_ensure(ctx, dX, (size_t)m * dims * 4);
  if (!rc) rc = dbgz_sobol_dev(ctx, m, dims, (const uint32_t *)dV.p, first, (uint32_t *)dX.p);
  if (!rc) {
    cudaMemcpyAsync(X, dX.p, (size_t)m * dims * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sobol_mat: copy back failed");
  }
  dbgz_release(dV); dbgz_release(dX);
  return rc;
}

// ---- the qmc_pnorm! path --------------------------------------------------
int dbgz_prepare(dbgz_ctx *ctx, int64_t d, const double *Sigma, const double *a, const double *b,
                 const dbgz_opts *opts, int qmc_type, int structure, int cdf_form,
                 const double *shifts, const uint64_t *ushifts, const uint32_t *sobol_dirnums,
                 int64_t sobol_first, dbgz_problem **out) {
  if (!out) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: out is NULL");
  *out = nullptr;
  if (!ctx || !Sigma || !a || !b)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: NULL Sigma/a/b");
  if (d < 2) return dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "prepare: d must be >= 2 (got %lld)", (long long)d);
  dbgz_opts o;
  if (opts) o = *opts; else dbgz_default_opts(&o);
  if (o.m < 1 || o.n_reps < 2 || o.max_pts < 0 || o.chol_block_size < 1 || o.chol_block_size2 < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: need m >= 1, n_reps >= 2, positive block sizes");
  if (qmc_type != DBGZ_QMC_RICHTMYER && qmc_type != DBGZ_QMC_SOBOL)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: bad qmc_type %d", qmc_type);
  if (structure != DBGZ_STRUCTURE_DENSE && structure != DBGZ_STRUCTURE_SPARSE)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: bad structure %d", structure);
  if (cdf_form != DBGZ_CDF_ERF && cdf_form != DBGZ_CDF_ERFC)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: bad cdf_form %d", cdf_form);
  if (qmc_type == DBGZ_QMC_RICHTMYER && !shifts)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: Richtmyer needs shifts");
  if (qmc_type == DBGZ_QMC_SOBOL) {
    if (!ushifts) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: Sobol needs ushifts");
    if (o.n_bits < 1 || o.n_bits > 32)
      return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: n_bits must be in 1..32");
    if (sobol_first < 0) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: sobol_first < 0");
  }
  // (Sigma itself is checked on the device after its upload: a host pass over
  // the d^2 entries cost about 1 ms at d = 1000)
  for (int64_t i = 0; i < d; ++i) {
    if (std::isnan(a[i]) || std::isnan(b[i]))
      return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "prepare: NaN bound at %lld", (long long)i);
    if (a[i] > b[i])
      return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "prepare: a[%lld] > b[%lld]", (long long)i, (long long)i);
  }
  if (qmc_type == DBGZ_QMC_RICHTMYER)
    for (int64_t i = 0; i < (d - 1) * o.n_reps; ++i)
      if (!(shifts[i] >= 0.0 && shifts[i] <= 1.0))
        return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "prepare: shifts must lie in [0,1]");
  cudaSetDevice(ctx->device);
  dbgz_problem *p = new (std::nothrow) dbgz_problem();
  if (!p) return dbgz_fail(ctx, DBGZ_ERR_OUT_OF_MEMORY, "prepare: host allocation");
  p->ctx = ctx;
  ctx->live_problems += 1;
  p->d = d;
  p->opts = o;
  p->qmc_type = qmc_type;
  p->structure = structure;
  p->cdf_form = cdf_form;
  p->sobol_first = sobol_first;
  p->lower_inf = true;
  for (int64_t i = 0; i < d; ++i) p->lower_inf = p->lower_inf && std::isinf(a[i]) && a[i] < 0;
  int rc = DBGZ_OK;
  const size_t nn = (size_t)d * d;
  const int64_t launches0 = ctx->launch_count;
  if (ctx->profiling) cudaEventRecord(ctx->ev[0], ctx->stream);
  DevBuf chk;  // first non-finite index of Sigma (UINT64_MAX: none)
  do {
    if ((rc = upload(ctx, p->U, Sigma, nn * 8))) break;
    if ((rc = dbgz_ensure(ctx, chk, 8))) break;
    if (cudaMemsetAsync(chk.p, 0xff, 8, ctx->stream) != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "prepare: memset failed");
      break;
    }
    k_first_nonfinite<<<(unsigned)std::min<int64_t>(((int64_t)nn + 255) / 256, 2048), 256, 0, ctx->stream>>>(
        (const double *)p->U.p, (int64_t)nn, (unsigned long long *)chk.p);
    dbgz_count_launch(ctx);
    // the factorisation runs on whatever Sigma holds (its loops are bounded);
    // a non-finite entry is reported before its rank
    auto sigma_ok = [&]() -> int {
      unsigned long long first = ~0ull;
      if (cudaMemcpy(&first, chk.p, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return dbgz_fail(ctx, DBGZ_ERR_CUDA, "prepare: %s", cudaGetErrorString(cudaGetLastError()));
      if (first != ~0ull)
        return dbgz_fail(ctx, DBGZ_ERR_NONFINITE_INPUT, "prepare: Sigma has a non-finite entry at %lld",
                         (long long)first);
      return DBGZ_OK;
    };
    if ((rc = upload(ctx, p->a, a, d * 8))) break;
    if ((rc = upload(ctx, p->b, b, d * 8))) break;
    if ((rc = dbgz_ensure(ctx, p->perm, d * 8))) break;
    if ((rc = dbgz_ensure(ctx, p->scale, d * 8))) break;
    if (structure == DBGZ_STRUCTURE_DENSE) {
      rc = dbgz_chol_genz_dev(ctx, d, (double *)p->U.p, (double *)p->a.p, (double *)p->b.p,
                              o.chol_block_size, o.chol_block_size2, 1024, 2048,
                              (int64_t *)p->perm.p, (double *)p->scale.p, &p->rank);
      if (rc) break;
      if ((rc = sigma_ok())) break;
      if (p->rank != d) {
        rc = dbgz_fail(ctx, DBGZ_ERR_RANK_DEFICIENT, "QMCData requires a full-rank Cholesky factorization. (rank %lld of %lld)",
                       (long long)p->rank, (long long)d);
        break;
      }
    } else {
      rc = dbgz_chol_classic_dev(ctx, d, (double *)p->U.p, (double *)p->a.p, (double *)p->b.p,
                                 o.chol_block_size, o.chol_block_size2, 1024, 2048,
                                 (double *)p->scale.p);
      if (rc) break;
      if ((rc = sigma_ok())) break;
      p->rank = d;
      std::vector<int64_t> id(d);
      for (int64_t i = 0; i < d; ++i) id[i] = i;
      if ((rc = upload(ctx, p->perm, id.data(), d * 8))) break;
    }
    if ((rc = dbgz_truncate_dev(ctx, d, (double *)p->U.p, 2.220446049250313e-16))) break;
    if (qmc_type == DBGZ_QMC_RICHTMYER) {
      std::vector<double> q(d - 1);
      dbgz_sqrt_primes(d - 1, q.data());
      std::vector<float> s32((d - 1) * o.n_reps);
      for (size_t i = 0; i < s32.size(); ++i) s32[i] = (float)shifts[i];
      if ((rc = upload(ctx, p->q, q.data(), (d - 1) * 8))) break;
      if ((rc = upload(ctx, p->shifts, shifts, (d - 1) * o.n_reps * 8))) break;
      if ((rc = upload(ctx, p->shifts32, s32.data(), s32.size() * 4))) break;
    } else {
      std::vector<uint32_t> V;
      const uint32_t *Vp = sobol_dirnums;
      if (!Vp) {
        V.resize((d - 1) * 32);
        if (dbgz_sobol_dirnums(d - 1, V.data()) != DBGZ_OK) {
          rc = dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "prepare: no Sobol table for %lld dims", (long long)(d - 1));
          break;
        }
        Vp = V.data();
      }
      if ((rc = upload(ctx, p->V, Vp, (d - 1) * 32 * 4))) break;
      if ((rc = upload(ctx, p->ushifts, ushifts, (d - 1) * o.n_reps * 8))) break;
    }
    if ((rc = dbgz_make_targets(p))) break;
    if (ctx->profiling) cudaEventRecord(ctx->ev[1], ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "prepare: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
  } while (0);
  dbgz_release(chk);
  if (rc != DBGZ_OK) {
    dbgz_problem_free(p);
    return rc;
  }
  if (ctx->profiling) {
    ctx->prof.prepare_ms = event_ms(ctx->ev[0], ctx->ev[1]);
    ctx->prof.prepare_launches = ctx->launch_count - launches0;
  }
  *out = p;
  return DBGZ_OK;
}

int dbgz_problem_free(dbgz_problem *p) {
  if (!p) return DBGZ_ERR_INVALID_ARGUMENT;
  if (p->ctx) {
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
  }
  DevBuf *bufs[] = {&p->U,     &p->a,       &p->b,       &p->perm,       &p->scale,   &p->q,         &p->shifts,
                    &p->shifts32, &p->V,   &p->ushifts, &p->tgt64,      &p->tgt32,   &p->U32,       &p->Uhi,
                    &p->Ulo,   &p->Utf,     &p->Ub,      &p->Ub32,       &p->Ubhi,    &p->Ublo,      &p->Ubtf,
                    &p->grad_buf, &p->yws, &p->partials, &p->reps,      &p->csc_colptr, &p->csc_row, &p->csc_val64,
                    &p->csc_val32, &p->cscb_colptr, &p->cscb_row, &p->cscb_val64, &p->cscb_val32};
  for (DevBuf *b : bufs) dbgz_release(*b);
  dbgz_drop_graphs(p);
  dbgz_release(p->drv_state);
  if (p->ctx) p->ctx->live_problems -= 1;
  delete p;
  return DBGZ_OK;
}

int dbgz_problem_set_cdf_form(dbgz_problem *p, int cdf_form) {
  if (!p) return DBGZ_ERR_INVALID_ARGUMENT;
  if (cdf_form != DBGZ_CDF_ERF && cdf_form != DBGZ_CDF_ERFC)
    return dbgz_fail(p->ctx, DBGZ_ERR_INVALID_ARGUMENT, "set_cdf_form: bad form %d", cdf_form);
  if (p->cdf_form != cdf_form) {
    p->c1_ready = false;
    dbgz_drop_graphs(p);
  }
  p->cdf_form = cdf_form;
  return DBGZ_OK;
}

int dbgz_problem_truncate_band(dbgz_problem *p, int64_t bandwidth) {
  if (!p || bandwidth < 1) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  cudaSetDevice(ctx->device);
  p->band = bandwidth;
  DBGZ_TRY(dbgz_band_dev(ctx, p->d, (double *)p->U.p, bandwidth));
  DevBuf *derived[] = {&p->U32, &p->Uhi,  &p->Ulo,  &p->Utf,  &p->Ub,         &p->Ub32,    &p->Ubhi,
                       &p->Ublo, &p->Ubtf, &p->csc_colptr, &p->csc_row, &p->csc_val64, &p->csc_val32,
                       &p->cscb_colptr, &p->cscb_row, &p->cscb_val64, &p->cscb_val32};
  for (DevBuf *b : derived) dbgz_release(*b);
  dbgz_drop_graphs(p);
  p->ldU = 0;
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return DBGZ_OK;
}

int dbgz_problem_factor(const dbgz_problem *p, double *U, int64_t *perm, double *a, double *b,
                        double *scale_vec, int64_t *rank) {
  if (!p) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  cudaSetDevice(ctx->device);
  const int64_t d = p->d;
  cudaStream_t st = ctx->stream;
  if (U) cudaMemcpyAsync(U, p->U.p, (size_t)d * d * 8, cudaMemcpyDeviceToHost, st);
  if (perm) cudaMemcpyAsync(perm, p->perm.p, d * 8, cudaMemcpyDeviceToHost, st);
  if (a) cudaMemcpyAsync(a, p->a.p, d * 8, cudaMemcpyDeviceToHost, st);
  if (b) cudaMemcpyAsync(b, p->b.p, d * 8, cudaMemcpyDeviceToHost, st);
  if (scale_vec) cudaMemcpyAsync(scale_vec, p->scale.p, d * 8, cudaMemcpyDeviceToHost, st);
  if (rank) *rank = p->rank;
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return DBGZ_OK;
}

int dbgz_first_dim_cdf(dbgz_problem *p) {
  if (p->c1_ready) return DBGZ_OK;
  dbgz_ctx *ctx = p->ctx;
  double a0, b0, u00;
  cudaMemcpyAsync(&a0, p->a.p, 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(&b0, p->b.p, 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(&u00, p->U.p, 8, cudaMemcpyDeviceToHost, ctx->stream);
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  // src/qmc.jl:800-809
  double arg_a = a0 / (u00 * std::sqrt(2.0));
  double arg_b = b0 / (u00 * std::sqrt(2.0));
  if (p->cdf_form == DBGZ_CDF_ERFC && p->structure == DBGZ_STRUCTURE_DENSE) {
    p->c1 = 0.5 * std::erfc(-arg_a);
    p->dc1 = 0.5 * (std::erfc(-arg_b) - std::erfc(-arg_a));
  } else {
    p->c1 = 0.5 * (1.0 + std::erf(arg_a));
    p->dc1 = 0.5 * (std::erf(arg_b) - std::erf(arg_a));
  }
  p->c1_ready = true;
  return DBGZ_OK;
}

static double sd_ref(const double *v, int64_t n, double mean) {
  double r = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double dd = v[i] - mean;
    r += dd * dd / (double)n;
  }
  return std::sqrt(r / (double)(n - 1));
}

int dbgz_pnorm(dbgz_problem *p, int precision, double *result, double *err, int64_t *n_pts,
               double *qmc_reps) {
  if (!p || !result || !err || !n_pts) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm: bad precision %d", precision);
  cudaSetDevice(ctx->device);
  const dbgz_opts &o = p->opts;
  const int64_t n_reps = o.n_reps, m = o.m;
  DBGZ_TRY(dbgz_first_dim_cdf(p));
  if (precision != DBGZ_PREC_FP64 && !p->U32.p) DBGZ_TRY(dbgz_make_U32(p));
  const int64_t tps = (m + 127) / 128;
  const int64_t n_tiles = tps * n_reps;
  DBGZ_TRY(dbgz_ensure(ctx, p->partials, sizeof(double) * n_tiles));
  DBGZ_TRY(dbgz_ensure(ctx, p->reps, sizeof(double) * n_reps));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(p->reps.p, 0, sizeof(double) * n_reps, ctx->stream));
  std::vector<double> reps(n_reps);
  PassArgs pa{};
  pa.d = p->d;
  pa.m = m;
  pa.n_reps = n_reps;
  pa.sobol_first = p->sobol_first;
  pa.n_bits = (int)o.n_bits;
  pa.qmc_type = p->qmc_type;
  pa.cdf_form = p->cdf_form;
  pa.c1 = p->c1;
  pa.dc1 = p->dc1;
  int64_t npts = 0;
  double res = 0.0, e = 0.0;
  bool first = true;
  const bool prof = ctx->profiling;
  dbgz_profile pr{};
  pr.prepare_ms = ctx->prof.prepare_ms;
  pr.prepare_launches = ctx->prof.prepare_launches;
  pr.grad_state_bytes = ctx->prof.grad_state_bytes;
  pr.grad_chunks = ctx->prof.grad_chunks;
  const int64_t launches0 = ctx->launch_count;
  if (prof) cudaEventRecord(ctx->ev[0], ctx->stream);
  while (true) {
    if (!first) p->gen_base += m;  // next_points! (src/qmc_generators.jl:119-131)
    pa.gen_base = p->gen_base;
    const int64_t l_before = ctx->launch_count;
    if (prof) cudaEventRecord(ctx->ev[2], ctx->stream);
    const bool sparse = p->structure == DBGZ_STRUCTURE_SPARSE;
    const bool tensor = !sparse && (precision == DBGZ_PREC_FP32_TF32 || precision == DBGZ_PREC_FP32_SPLIT_BF16);
    if (sparse)
      DBGZ_TRY(dbgz_loop_sparse(p, pa, precision, (double *)p->partials.p, n_tiles));
    else if (tensor)
      DBGZ_TRY(dbgz_loop_umma(p, pa, precision, (double *)p->partials.p, n_tiles));
    else
      DBGZ_TRY(dbgz_loop_simt(p, pa, precision, (double *)p->partials.p, n_tiles));
    if (prof) cudaEventRecord(ctx->ev[3], ctx->stream);
    pr.loop_launches += ctx->launch_count - l_before;
    if (prof) cudaEventRecord(ctx->ev[4], ctx->stream);
    DBGZ_TRY(dbgz_finalize_pass(p, (const double *)p->partials.p, tps, npts, m, (double *)p->reps.p));
    if (prof) cudaEventRecord(ctx->ev[5], ctx->stream);
    DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(reps.data(), p->reps.p, sizeof(double) * n_reps,
                                       cudaMemcpyDeviceToHost, ctx->stream));
    int dev_status = 0;
    if (tensor)
      DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(&dev_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost,
                                         ctx->stream));
    if (prof) cudaEventRecord(ctx->ev[1], ctx->stream);
    DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (dev_status != 0)
      return dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm: a bounded wait in the tensor-core loop gave up (status %d)",
                       dev_status);
    if (prof) {
      pr.loop_ms += event_ms(ctx->ev[2], ctx->ev[3]);
      pr.finalize_ms += event_ms(ctx->ev[4], ctx->ev[5]);
    }
    res = 0.0;
    for (int64_t k = 0; k < n_reps; ++k) res += reps[k];
    res /= (double)n_reps;
    e = 3.0 * sd_ref(reps.data(), n_reps, res);
    npts += m;
    first = false;
    if (npts >= o.max_pts || e < o.max_abs_err) break;  // src/qmc.jl:824, :835
    if (!(e > o.max_abs_err)) break;
  }
  if (prof) {
    pr.pnorm_ms = event_ms(ctx->ev[0], ctx->ev[1]);
    pr.kernel_launches = ctx->launch_count - launches0;
    ctx->prof = pr;
  }
  *result = res;
  *err = e;
  *n_pts = npts;
  if (qmc_reps) std::memcpy(qmc_reps, reps.data(), sizeof(double) * n_reps);
  return DBGZ_OK;
}

int dbgz_pnorm_logw(dbgz_problem *p, int precision, double *logw, double *qmc_reps) {
  if (!p || !logw) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_logw: bad precision %d", precision);
  cudaSetDevice(ctx->device);
  const dbgz_opts &o = p->opts;
  const int64_t n_reps = o.n_reps, m = o.m;
  DBGZ_TRY(dbgz_first_dim_cdf(p));
  if (precision != DBGZ_PREC_FP64 && !p->U32.p) DBGZ_TRY(dbgz_make_U32(p));
  const int64_t tps = (m + 127) / 128;
  const int64_t n_tiles = tps * n_reps;
  DBGZ_TRY(dbgz_ensure(ctx, p->partials, sizeof(double) * n_tiles));
  DBGZ_TRY(dbgz_ensure(ctx, p->reps, sizeof(double) * n_reps));
  DevBuf lw;  // one double per sample, [tile * 128 + row]; back to the pool at the end
  struct Release {
    DevBuf &b;
    ~Release() { dbgz_release(b); }
  } release_lw{lw};
  DBGZ_TRY(dbgz_ensure(ctx, lw, sizeof(double) * (size_t)n_tiles * 128));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(p->reps.p, 0, sizeof(double) * n_reps, ctx->stream));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  PassArgs pa{};
  pa.kind = kLoopLogWeight;
  pa.d = p->d;
  pa.m = m;
  pa.n_reps = n_reps;
  pa.sobol_first = p->sobol_first;
  pa.n_bits = (int)o.n_bits;
  pa.qmc_type = p->qmc_type;
  pa.cdf_form = p->cdf_form;
  pa.c1 = p->c1;
  pa.dc1 = p->dc1;
  pa.gen_base = p->gen_base;
  pa.grad.N = n_tiles * 128;
  pa.grad.p = (double *)lw.p;
  pa.grad.dc1 = p->dc1;
  const bool sparse = p->structure == DBGZ_STRUCTURE_SPARSE;
  const bool tensor = !sparse && (precision == DBGZ_PREC_FP32_TF32 || precision == DBGZ_PREC_FP32_SPLIT_BF16);
  if (sparse)
    DBGZ_TRY(dbgz_loop_sparse(p, pa, precision, (double *)p->partials.p, n_tiles));
  else if (tensor)
    DBGZ_TRY(dbgz_loop_umma(p, pa, precision, (double *)p->partials.p, n_tiles));
  else
    DBGZ_TRY(dbgz_loop_simt(p, pa, precision, (double *)p->partials.p, n_tiles));
  DBGZ_TRY(dbgz_finalize_pass(p, (const double *)p->partials.p, tps, 0, m, (double *)p->reps.p));
  // the shift-major tile order gives point j of shift k at k * tps * 128 + j
  DBGZ_CUDA_TRY(ctx, cudaMemcpy2DAsync(logw, sizeof(double) * (size_t)m, lw.p, sizeof(double) * (size_t)tps * 128,
                                       sizeof(double) * (size_t)m, (size_t)n_reps, cudaMemcpyDeviceToHost,
                                       ctx->stream));
  std::vector<double> reps(n_reps);
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(reps.data(), p->reps.p, sizeof(double) * n_reps, cudaMemcpyDeviceToHost,
                                     ctx->stream));
  int dev_status = 0;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(&dev_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (dev_status != 0)
    return dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm_logw: a bounded wait in the tensor-core loop gave up");
  if (qmc_reps) std::memcpy(qmc_reps, reps.data(), sizeof(double) * n_reps);
  return DBGZ_OK;
}

}  // extern "C"

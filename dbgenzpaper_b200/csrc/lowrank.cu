// lowrank.cu -- dbgz_cholesky_rowmax and dbgz_adapt_low_rank: the rest of
// the reference's factorisation family (src/cholesky.jl:24-123, 244-432).
// qmc_pnorm! calls neither; they are the tools a caller uses on a singular
// covariance.
//
// adapt_low_rank! walks the dependent columns rank+1..n of a rank-r factor:
// a column with no entry above eps1 in rows 1..r goes to the end; any other
// is scaled by its last such entry (the "level" i_j; the bounds swap when it
// is negative) and moved to the end of the block of level i_j.  Which column
// goes where depends only on the levels, and a column's level is fixed
// before anything moves it, so here the levels and pivots of all columns
// are found at once on the device, the reference's sequence of swaps and
// block shifts is replayed on column indices on the host, and one gather
// kernel writes every column to its final place, scaled: the same values
// (one IEEE multiply by the same reciprocal per entry) without moving any
// column more than once.
#include <cmath>
#include <vector>

#include "internal.cuh"

namespace {

// level[j] (1-based, 0: none) = last row i < rank with |M[i, j]| > eps1, and
// piv[j] = M[level - 1, j], for the columns j in [rank, n); one CTA each
__global__ void k_adapt_levels(const double *M, int64_t nr, int64_t rank, double eps1, int64_t *level,
                               double *piv) {
  const int64_t j = rank + blockIdx.x;
  __shared__ int64_t best[32];
  int64_t b = -1;
  const int64_t top = rank < nr ? rank : nr;
  for (int64_t i = threadIdx.x; i < top; i += blockDim.x)
    if (fabs(M[j * nr + i]) > eps1) b = i > b ? i : b;
  for (int o = 16; o > 0; o >>= 1) {
    const int64_t v = __shfl_down_sync(0xffffffffu, b, o);
    b = v > b ? v : b;
  }
  if ((threadIdx.x & 31) == 0) best[threadIdx.x >> 5] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = best[w] > b ? best[w] : b;
    level[j - rank] = b + 1;
    piv[j - rank] = b >= 0 ? M[j * nr + b] : 0.0;
  }
}

// Mout[:, c] = Min[:, src[c]], rows below lvl[c] scaled by inv[c]
// (lvl[c] = 0: copied as is)
__global__ void k_adapt_gather(const double *Min, int64_t nr, const int64_t *src, const int64_t *lvl,
                               const double *inv, double *Mout) {
  const int64_t c = blockIdx.y;
  const int64_t s = src[c], L = lvl[c];
  const double f = inv[c];
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nr; r += (int64_t)gridDim.x * blockDim.x) {
    const double v = Min[s * nr + r];
    Mout[c * nr + r] = r < L ? v * f : v;
  }
}

}  // namespace

extern "C" {

int dbgz_cholesky_rowmax(dbgz_ctx *ctx, int64_t d, double *M, double *a, double *b, int64_t bs1, int64_t bs2,
                         int64_t bs3, int64_t bs4, int64_t *perm, double *scale_vec, int64_t *rank) {
  if (!ctx || !M || !a || !b || !perm || !scale_vec || !rank || d < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "cholesky_rowmax: bad argument");
  cudaSetDevice(ctx->device);
  DevBuf dM, da, db, dp, ds;
  const size_t nn = (size_t)d * d;
  int rc = DBGZ_OK;
  if ((rc = dbgz_ensure(ctx, dM, nn * 8)) || (rc = dbgz_ensure(ctx, da, d * 8)) || (rc = dbgz_ensure(ctx, db, d * 8)) ||
      (rc = dbgz_ensure(ctx, dp, d * 8)) || (rc = dbgz_ensure(ctx, ds, d * 8)))
    goto done;
  if (cudaMemcpyAsync(dM.p, M, nn * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
      cudaMemcpyAsync(da.p, a, d * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
      cudaMemcpyAsync(db.p, b, d * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_rowmax: upload failed");
    goto done;
  }
  rc = dbgz_chol_rowmax_dev(ctx, d, (double *)dM.p, (double *)da.p, (double *)db.p, bs1, bs2, bs3, bs4,
                            (int64_t *)dp.p, (double *)ds.p, rank);
  if (rc) goto done;
  cudaMemcpyAsync(M, dM.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(a, da.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(b, db.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(perm, dp.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(scale_vec, ds.p, d * 8, cudaMemcpyDeviceToHost, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_rowmax: copy back failed");
done:
  dbgz_release(dM);
  dbgz_release(da);
  dbgz_release(db);
  dbgz_release(dp);
  dbgz_release(ds);
  return rc;
}

int dbgz_adapt_low_rank(dbgz_ctx *ctx, int64_t nr, int64_t n, double *M, double *a, double *b, int64_t rank,
                        int64_t *perm, double eps1, int64_t *k_js, int64_t *k_0) {
  if (!ctx || !M || !a || !b || !perm || !k_0 || nr < 0 || n < 0 || rank < 0 || rank > n || (rank > 0 && !k_js))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "adapt_low_rank: bad argument");
  cudaSetDevice(ctx->device);
  const int64_t nd = n - rank;  // dependent columns
  for (int64_t i = 0; i < rank; ++i) k_js[i] = i + 1;
  *k_0 = 0;
  if (nd == 0) return DBGZ_OK;
  const size_t mb = (size_t)nr * (size_t)n * 8;
  DevBuf dM, dO, dl, dpv, dsrc, dlv, dinv;
  int rc = DBGZ_OK;
  std::vector<int64_t> level(nd), col(n), lvl_at(n, 0);
  std::vector<double> piv(nd), inv_at(n, 1.0);
  if ((rc = dbgz_ensure(ctx, dM, mb + 8)) || (rc = dbgz_ensure(ctx, dO, mb + 8)) ||
      (rc = dbgz_ensure(ctx, dl, 8 * (size_t)nd)) || (rc = dbgz_ensure(ctx, dpv, 8 * (size_t)nd)) ||
      (rc = dbgz_ensure(ctx, dsrc, 8 * (size_t)n)) || (rc = dbgz_ensure(ctx, dlv, 8 * (size_t)n)) ||
      (rc = dbgz_ensure(ctx, dinv, 8 * (size_t)n)))
    goto done;
  if (cudaMemcpyAsync(dM.p, M, mb, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "adapt_low_rank: upload failed");
    goto done;
  }
  k_adapt_levels<<<(unsigned)nd, 256, 0, ctx->stream>>>((const double *)dM.p, nr, rank, eps1, (int64_t *)dl.p,
                                                       (double *)dpv.p);
  dbgz_count_launch(ctx);
  cudaMemcpyAsync(level.data(), dl.p, 8 * (size_t)nd, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(piv.data(), dpv.p, 8 * (size_t)nd, cudaMemcpyDeviceToHost, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "adapt_low_rank: level scan failed");
    goto done;
  }
  {
    // the reference's loop (src/cholesky.jl:38-120) on column indices
    for (int64_t c = 0; c < n; ++c) col[c] = c;
    std::vector<int64_t> kj(rank);
    for (int64_t i = 0; i < rank; ++i) kj[i] = i + 1;
    int64_t k0 = 0, j = rank + 1, n_active = n;  // 1-based as in the reference
    while (j <= n_active) {
      const int64_t c = col[j - 1];
      const int64_t i_j = level[c - rank];
      if (i_j == 0) {
        if (j != n_active) {
          std::swap(col[j - 1], col[n_active - 1]);
          std::swap(a[j - 1], a[n_active - 1]);
          std::swap(b[j - 1], b[n_active - 1]);
          std::swap(perm[j - 1], perm[n_active - 1]);
        }
        ++k0;
        --n_active;
        continue;
      }
      const double m_ij = piv[c - rank];
      const bool is_neg = m_ij < 0.0;
      const double inv_m = 1.0 / m_ij;
      lvl_at[c] = i_j;
      inv_at[c] = inv_m;
      a[j - 1] *= inv_m;
      b[j - 1] *= inv_m;
      if (is_neg) std::swap(a[j - 1], b[j - 1]);
      const int64_t pos = kj[i_j - 1] + 1;
      if (j != pos) {
        const int64_t vc = col[j - 1], vp = perm[j - 1];
        const double va = a[j - 1], vb = b[j - 1];
        for (int64_t q = j; q >= pos + 1; --q) {
          col[q - 1] = col[q - 2];
          a[q - 1] = a[q - 2];
          b[q - 1] = b[q - 2];
          perm[q - 1] = perm[q - 2];
        }
        col[pos - 1] = vc;
        a[pos - 1] = va;
        b[pos - 1] = vb;
        perm[pos - 1] = vp;
      }
      for (int64_t k = i_j; k <= rank; ++k) kj[k - 1] += 1;
      ++j;
    }
    for (int64_t i = 0; i < rank; ++i) k_js[i] = kj[i];
    *k_0 = k0;
  }
  {
    std::vector<int64_t> lv(n);
    std::vector<double> iv(n);
    for (int64_t c = 0; c < n; ++c) {
      lv[c] = lvl_at[col[c]];
      iv[c] = inv_at[col[c]];
    }
    cudaMemcpyAsync(dsrc.p, col.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dlv.p, lv.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dinv.p, iv.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    if (nr > 0) {
      const dim3 g((unsigned)std::max<int64_t>(1, std::min<int64_t>((nr + 255) / 256, 64)), (unsigned)n);
      k_adapt_gather<<<g, 256, 0, ctx->stream>>>((const double *)dM.p, nr, (const int64_t *)dsrc.p,
                                                  (const int64_t *)dlv.p, (const double *)dinv.p, (double *)dO.p);
      dbgz_count_launch(ctx);
      cudaMemcpyAsync(M, dO.p, mb, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "adapt_low_rank: gather failed");
  }
done:
  dbgz_release(dM);
  dbgz_release(dO);
  dbgz_release(dl);
  dbgz_release(dpv);
  dbgz_release(dsrc);
  dbgz_release(dlv);
  dbgz_release(dinv);
  return rc;
}

}  // extern "C"

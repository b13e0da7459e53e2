// chol_adjoint.cu -- dbgz_problem_sigma_adjoint: dP/dSigma from the factor
// gradient, through the pivoted Cholesky and the correlation scaling.
//
// No counterpart in the reference (it has no gradient).  The forward chain
// of dbgz_prepare is
//   s_i = sqrt(Sigma_ii),  R = D^-1 Sigma D^-1,  a'_i = a_i / s_i (b' alike),
//   R[pi, pi] = U' U (Genz pivoting, permutation pi held fixed),
//   a''_t = a'_{pi t},  P = P(U, a'', b'').
// With L = U' and Lbar = Ubar', the Cholesky adjoint (Murray 2016, "
// Differentiation of the Cholesky decomposition") is
//   S = L^-T Phi(L' Lbar) L^-1 = U^-1 Phi(U Ubar') U^-T,
// Phi = lower triangle with the diagonal halved, and G = (S + S')/2 is the
// gradient with respect to the permuted correlation matrix for symmetric
// perturbations.  The scaling then gives, in the original order,
//   dP/dSigma_ij = G_ij / (s_i s_j)                                  (i != j)
//   dP/dSigma_ii = (G_ii - sum_j G_ij R_ij - (abar'' a'' + bbar'' b'')/2) / s_i^2
// where abar''_t = dP/da_{pi t} * s_{pi t} is the gradient with respect to
// the scaled bound.  The dense FP64 linear algebra runs in this library's own
// kernels (dense64.cuh) on the context's stream:
//   M = Phi(U Ubar')            one GEMM over k >= max(i, j), lower triangle
//                               written with the halved diagonal;
//   V = U^-1                    triangular inverse;
//   S = (V M) V'                two GEMMs over the triangles' nonzero blocks;
//   R = U'U                     one GEMM over k <= min(i, j).
#include <cmath>
#include <vector>

#include "dense64.cuh"
#include "internal.cuh"

namespace {

// Uc = triu(U); T1 = Ubar' restricted to the lower triangle (Ubar's upper
// triangle transposed)
__global__ void k_adj_prepare(const double *U, const double *Ubar, int64_t d, double *Uc, double *T1) {
  const int64_t j = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d; i += (int64_t)gridDim.x * blockDim.x) {
    Uc[j * d + i] = i <= j ? U[j * d + i] : 0.0;
    T1[j * d + i] = i >= j ? Ubar[i * d + j] : 0.0;  // T1[i, j] = Ubar[j, i]
  }
}

// r_i = sum_j G_ij R_ij with G = (S + S')/2 and R = U'U symmetric:
// r = (row sums + column sums of S o R) / 2.  Row sums: one thread per row,
// ascending j (coalesced over i); column sums: one warp per column
// (contiguous), a fixed lane order and shuffle tree.
__global__ void k_adj_rowsum(const double *S, const double *R, int64_t d, double *rs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= d) return;
  // the same ascending chain, its operands loaded 16 at a time ahead of it
  double acc = 0.0;
  int64_t j = 0;
  for (; j + 16 <= d; j += 16) {
    double x[16], y[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x[u] = S[(j + u) * d + i];
      y[u] = R[(j + u) * d + i];
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) acc = fma(x[u], y[u], acc);
  }
  for (; j < d; ++j) acc = fma(S[j * d + i], R[j * d + i], acc);
  rs[i] = acc;
}
__global__ void k_adj_colsum(const double *S, const double *R, int64_t d, const double *rs, double *r) {
  const int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= d) return;
  double acc = 0.0;
  for (int64_t j = lane; j < d; j += 32) acc = fma(S[i * d + j], R[i * d + j], acc);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) r[i] = 0.5 * (rs[i] + acc);
}

// out[pi i, pi j] from the permuted-coordinate G, scaling and bound terms
__global__ void k_adj_scatter(const double *S, const double *r, const int64_t *perm, const double *scale,
                              const double *ap, const double *bp, const double *abar, const double *bbar, int64_t d,
                              double *out) {
  const int64_t j = blockIdx.y;
  const int64_t oj = perm[j];
  const double sj = scale[oj];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t oi = perm[i];
    const double si = scale[oi];
    const double g = 0.5 * (S[j * d + i] + S[i * d + j]);
    double v;
    if (i != j) {
      v = g / (si * sj);
    } else {
      // bound terms: gradient w.r.t. the scaled bound times the bound
      // (zero where the gradient is zero, e.g. at an infinite bound)
      const double ga = abar ? abar[oi] * si : 0.0, gb = bbar ? bbar[oi] * si : 0.0;
      const double ta = ga != 0.0 ? ga * ap[i] : 0.0, tb = gb != 0.0 ? gb * bp[i] : 0.0;
      v = (g - r[i] - 0.5 * (ta + tb)) / (si * si);
    }
    out[oj * d + oi] = v;
  }
}

}  // namespace

// Device inputs (dU: d x d FP64 factor gradient, upper triangle read; da,
// db: original-order bound gradients or NULL); enqueues the D2H copy of the
// result into host_out on the context's stream without waiting for it.
int dbgz_sigma_adjoint_dev(dbgz_problem *p, const double *dU, const double *da, const double *db,
                           double *host_out) {
  dbgz_ctx *ctx = p->ctx;
  if (p->structure != DBGZ_STRUCTURE_DENSE)
    return dbgz_fail(ctx, DBGZ_ERR_UNSUPPORTED, "sigma_adjoint: the adjoint is built for the dense structure");
  const int64_t d = p->d;
  const size_t nn = (size_t)d * d;
  cudaStream_t st = ctx->stream;
  DevBuf w;
  DBGZ_TRY(dbgz_ensure(ctx, w, 8 * (6 * nn + 2 * (size_t)d) + 4096));
  double *Uc = (double *)w.p, *T1 = Uc + nn, *M = T1 + nn, *R = M + nn, *V = R + nn, *X = V + nn, *r = X + nn,
         *rs = r + d;
  int rc = DBGZ_OK;
  do {
    const dim3 g2((unsigned)((d + 255) / 256), (unsigned)d);
    k_adj_prepare<<<g2, 256, 0, st>>>((const double *)p->U.p, dU, d, Uc, T1);
    dbgz_count_launch(ctx);
    int nl = 0;
    // M's tiles strictly above the diagonal are not written by the first GEMM
    cudaError_t ce = cudaMemsetAsync(M, 0, 8 * nn, st);
    dense64::GemmArgs g;
    // M = Phi(Uc T1): Uc[i,k] = 0 for k < i, T1[k,j] = 0 for k < j
    g.m = g.n = g.k = d;
    g.A = Uc; g.lda = d; g.B = T1; g.ldb = d; g.C = M; g.ldc = d;
    g.kmin_row = g.kmin_col = 1;
    g.out = dense64::kOutLowerPhi;
    if (ce == cudaSuccess) ce = dense64::gemm64<false, false>(g, st, &nl);
    // V = U^-1
    if (ce == cudaSuccess) ce = dense64::trinv64(Uc, d, V, st, &nl);
    // X = V M: V[i,k] = 0 for k < i, M[k,j] = 0 for k < j
    if (ce == cudaSuccess) {
      g = dense64::GemmArgs{};
      g.m = g.n = g.k = d;
      g.A = V; g.lda = d; g.B = M; g.ldb = d; g.C = X; g.ldc = d;
      g.kmin_row = g.kmin_col = 1;
      ce = dense64::gemm64<false, false>(g, st, &nl);
    }
    // S = X V' (into M): V'[k,j] = V[j,k] = 0 for k < j
    if (ce == cudaSuccess) {
      g = dense64::GemmArgs{};
      g.m = g.n = g.k = d;
      g.A = X; g.lda = d; g.B = V; g.ldb = d; g.C = M; g.ldc = d;
      g.kmin_col = 1;
      ce = dense64::gemm64<false, true>(g, st, &nl);
    }
    // R = Uc' Uc, the permuted correlation matrix: Uc[k,i] = 0 for k > i
    if (ce == cudaSuccess) {
      g = dense64::GemmArgs{};
      g.m = g.n = g.k = d;
      g.A = Uc; g.lda = d; g.B = Uc; g.ldb = d; g.C = R; g.ldc = d;
      g.kmax_row = g.kmax_col = 1;
      ce = dense64::gemm64<true, false>(g, st, &nl);
    }
    for (int i = 0; i < nl; ++i) dbgz_count_launch(ctx);
    if (ce != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sigma_adjoint: dense kernel launch failed (%s)", cudaGetErrorString(ce));
      break;
    }
    k_adj_rowsum<<<(unsigned)((d + 31) / 32), 32, 0, st>>>(M, R, d, rs);  // a warp per 32 rows: more SMs
    dbgz_count_launch(ctx);
    k_adj_colsum<<<(unsigned)((d + 7) / 8), 256, 0, st>>>(M, R, d, rs, r);
    dbgz_count_launch(ctx);
    // T1 is free now: the result in original order
    k_adj_scatter<<<g2, 256, 0, st>>>(M, r, (const int64_t *)p->perm.p, (const double *)p->scale.p,
                                      (const double *)p->a.p, (const double *)p->b.p, da, db, d, T1);
    dbgz_count_launch(ctx);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(host_out, T1, 8 * nn, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sigma_adjoint: launch or copy failed");
      break;
    }
  } while (0);
  dbgz_release(w);  // stream-ordered: a later user of the block runs after the copy
  return rc;
}

extern "C" int dbgz_problem_sigma_adjoint(dbgz_problem *p, const double *dP_dU, const double *dP_da,
                                          const double *dP_db, double *dP_dSigma) {
  if (!p || !dP_dU || !dP_dSigma) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  cudaSetDevice(ctx->device);
  const int64_t d = p->d;
  const size_t nn = (size_t)d * d;
  cudaStream_t st = ctx->stream;
  DevBuf in;
  DBGZ_TRY(dbgz_ensure(ctx, in, 8 * (nn + 2 * (size_t)d) + 1024));
  double *Ubar = (double *)in.p, *abar = Ubar + nn, *bbar = abar + d;
  const bool prof = ctx->profiling;
  if (prof) cudaEventRecord(ctx->ev[0], st);
  int rc = DBGZ_OK;
  if (cudaMemcpyAsync(Ubar, dP_dU, 8 * nn, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      (dP_da && cudaMemcpyAsync(abar, dP_da, 8 * d, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      (dP_db && cudaMemcpyAsync(bbar, dP_db, 8 * d, cudaMemcpyHostToDevice, st) != cudaSuccess))
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sigma_adjoint: upload failed");
  if (rc == DBGZ_OK)
    rc = dbgz_sigma_adjoint_dev(p, Ubar, dP_da ? abar : nullptr, dP_db ? bbar : nullptr, dP_dSigma);
  if (prof) cudaEventRecord(ctx->ev[1], st);
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == DBGZ_OK)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sigma_adjoint: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc == DBGZ_OK && prof) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    ctx->prof.sigma_adjoint_ms = ms;
  }
  dbgz_release(in);
  return rc;
}

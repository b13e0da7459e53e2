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
// the scaled bound.  Dense FP64 linear algebra (TRMM, two TRSMs, one GEMM)
// is cuBLAS on the context's stream; the rest are small kernels here.
#include <cublas_v2.h>

#include <cmath>
#include <vector>

#include "internal.cuh"

int dbgz_get_cublas(dbgz_ctx *ctx, cublasHandle_t *out);  // grad.cu

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

// M <- Phi(M): lower triangle, diagonal halved, upper triangle zero
__global__ void k_adj_phi(double *M, int64_t d) {
  const int64_t j = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d; i += (int64_t)gridDim.x * blockDim.x) {
    double &v = M[j * d + i];
    v = i > j ? v : (i == j ? 0.5 * v : 0.0);
  }
}

// r_i = sum_j G_ij R_ij with G = (S + S')/2, one thread per row, ascending j
__global__ void k_adj_rowsum(const double *S, const double *R, int64_t d, double *r) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= d) return;
  double acc = 0.0;
  for (int64_t j = 0; j < d; ++j) acc += 0.5 * (S[j * d + i] + S[i * d + j]) * R[j * d + i];
  r[i] = acc;
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
  DBGZ_TRY(dbgz_ensure(ctx, w, 8 * (4 * nn + (size_t)d) + 4096));
  double *Uc = (double *)w.p, *T1 = Uc + nn, *M = T1 + nn, *R = M + nn, *r = R + nn;
  int rc = DBGZ_OK;
  do {
    cublasHandle_t h;
    if ((rc = dbgz_get_cublas(ctx, &h))) break;
    const dim3 g2((unsigned)((d + 255) / 256), (unsigned)d);
    k_adj_prepare<<<g2, 256, 0, st>>>((const double *)p->U.p, dU, d, Uc, T1);
    dbgz_count_launch(ctx);
    const double one = 1.0, zero = 0.0;
    const int n = (int)d;
    cublasStatus_t cs;
    // M = U Ubar'
    cs = cublasDtrmm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, n, &one, Uc,
                     n, T1, n, M, n);
    if (cs == CUBLAS_STATUS_SUCCESS) {
      k_adj_phi<<<g2, 256, 0, st>>>(M, d);
      dbgz_count_launch(ctx);
      // S = U^-1 Phi(M) U^-T, in place
      cs = cublasDtrsm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, n, &one,
                       Uc, n, M, n);
    }
    if (cs == CUBLAS_STATUS_SUCCESS)
      cs = cublasDtrsm(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, n, n, &one,
                       Uc, n, M, n);
    // R = U' U, the permuted correlation matrix
    if (cs == CUBLAS_STATUS_SUCCESS)
      cs = cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, n, n, n, &one, Uc, n, Uc, n, &zero, R, n);
    if (cs != CUBLAS_STATUS_SUCCESS) {
      rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "sigma_adjoint: cuBLAS failed (%d)", (int)cs);
      break;
    }
    k_adj_rowsum<<<(unsigned)((d + 127) / 128), 128, 0, st>>>(M, R, d, r);
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

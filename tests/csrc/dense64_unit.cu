// dense64_unit.cu -- test-only C entry points over the FP64 dense kernels of
// the gradient path (dbgenzpaper_b200/csrc/dense64.cuh): one GEMM or one
// triangular inverse on host arrays.  Built by tests/test_gpu_dense64.py.
#include <cuda_runtime.h>
#include <cstdint>

#include "../../dbgenzpaper_b200/csrc/dense64.cuh"

extern "C" int dense64_gemm(int ta, int tb, int64_t m, int64_t n, int64_t k, const double *A, int64_t lda,
                            const double *B, int64_t ldb, double *C, int64_t ldc, int kmin_row, int kmin_col,
                            int kmax_row, int kmax_col, int out, int accumulate, int splits) {
  const int64_t ka = ta ? m : k, ca = ta ? k : m;  // stored A: lda x (ta ? m : k)
  const size_t a_bytes = sizeof(double) * (size_t)lda * (size_t)(ta ? m : k);
  const size_t b_bytes = sizeof(double) * (size_t)ldb * (size_t)(tb ? k : n);
  const size_t c_bytes = sizeof(double) * (size_t)ldc * (size_t)n;
  (void)ka;
  (void)ca;
  double *dA, *dB, *dC, *dP = nullptr;
  if (cudaMalloc(&dA, a_bytes) || cudaMalloc(&dB, b_bytes) || cudaMalloc(&dC, c_bytes)) return 1;
  cudaMemcpy(dA, A, a_bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, B, b_bytes, cudaMemcpyHostToDevice);
  cudaMemcpy(dC, C, c_bytes, cudaMemcpyHostToDevice);
  dense64::GemmArgs g;
  g.m = m; g.n = n; g.k = k; g.A = dA; g.lda = lda; g.B = dB; g.ldb = ldb; g.C = dC; g.ldc = ldc;
  g.kmin_row = kmin_row; g.kmin_col = kmin_col; g.kmax_row = kmax_row; g.kmax_col = kmax_col;
  g.out = out; g.accumulate = accumulate; g.splits = splits;
  const size_t pb = dense64::gemm64_partial_bytes(g);
  if (pb && cudaMalloc(&dP, pb)) return 1;
  g.partial = dP;
  cudaError_t e;
  if (ta && tb) e = dense64::gemm64<true, true>(g, 0);
  else if (ta) e = dense64::gemm64<true, false>(g, 0);
  else if (tb) e = dense64::gemm64<false, true>(g, 0);
  else e = dense64::gemm64<false, false>(g, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaMemcpy(C, dC, c_bytes, cudaMemcpyDeviceToHost);
  cudaFree(dA); cudaFree(dB); cudaFree(dC);
  if (dP) cudaFree(dP);
  return e == cudaSuccess ? 0 : 2;
}

extern "C" int dense64_trinv(int64_t d, const double *U, double *X) {
  double *dU, *dX;
  const size_t bytes = sizeof(double) * (size_t)d * d;
  if (cudaMalloc(&dU, bytes) || cudaMalloc(&dX, bytes)) return 1;
  cudaMemcpy(dU, U, bytes, cudaMemcpyHostToDevice);
  cudaError_t e = dense64::trinv64(dU, d, dX, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaMemcpy(X, dX, bytes, cudaMemcpyDeviceToHost);
  cudaFree(dU); cudaFree(dX);
  return e == cudaSuccess ? 0 : 2;
}

// Evaluates the library's FP32 tail mass and inverse normal
// (dbgenzpaper_b200/csrc/normal32.cuh) on host-given points, for
// tests/test_gpu_special.py.
#include <cuda_runtime.h>
#include "../../dbgenzpaper_b200/csrc/normal32.cuh"

__global__ void k_tail(const float *x, float *out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = dbgz::tail_mass_f32(x[i]);
}

__global__ void k_phiinv(const float *x, float *out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = dbgz::phi_inv_lower_f32(x[i]);
}

extern "C" int phi_inv_eval(const float *x, float *out, int n) {
  float *dx = nullptr, *dout = nullptr;
  if (cudaMalloc(&dx, sizeof(float) * n) != cudaSuccess) return 1;
  if (cudaMalloc(&dout, sizeof(float) * n) != cudaSuccess) { cudaFree(dx); return 1; }
  cudaMemcpy(dx, x, sizeof(float) * n, cudaMemcpyHostToDevice);
  k_phiinv<<<(n + 255) / 256, 256>>>(dx, dout, n);
  cudaError_t e = cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  return e == cudaSuccess ? 0 : 2;
}

extern "C" int tail_mass_eval(const float *x, float *out, int n) {
  float *dx = nullptr, *dout = nullptr;
  if (cudaMalloc(&dx, sizeof(float) * n) != cudaSuccess) return 1;
  if (cudaMalloc(&dout, sizeof(float) * n) != cudaSuccess) { cudaFree(dx); return 1; }
  cudaMemcpy(dx, x, sizeof(float) * n, cudaMemcpyHostToDevice);
  k_tail<<<(n + 255) / 256, 256>>>(dx, dout, n);
  cudaError_t e = cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  return e == cudaSuccess ? 0 : 2;
}

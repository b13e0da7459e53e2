// umma_unit.cu -- test-only kernel checking the tcgen05/TMA conventions the
// tensor-core loop relies on, in isolation: one CTA computes
//   D[128 x N] = A[128 x 32] * B[N x 32]^T
// with A written by threads into the swizzled K-major layout, B loaded by
// TMA with the matching swizzle, the product on tcgen05 (split BF16: three
// products hi*hi + hi*lo + lo*hi; or TF32: one product), a B row offset and
// a TMEM column offset as the loop's second MMA uses, and the accumulator
// read back with tcgen05.ld.  Built by tests/test_gpu_umma.py.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../dbgenzpaper_b200/csrc/sm100.cuh"

using namespace sm100;

namespace {

struct __align__(64) Params {
  CUtensorMap tm_b[2];
  const float *A;  // 128 x 32 row-major
  float *D;        // 128 x N row-major
  int N, b_row_off, d_col_off, mode;  // mode 2 = split bf16, 1 = tf32
  int *status;
};

constexpr int kSmem = 4 * 16384 + 4096;

__global__ void __launch_bounds__(160) k_umma_unit(const __grid_constant__ Params P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *A0 = sm, *A1 = sm + 16384;           // A parts (hi, lo) or tf32
  unsigned char *B0 = sm + 32768, *B1 = sm + 49152;   // B parts
  uint64_t *bars = (uint64_t *)(sm + 65536);
  uint32_t *tbase = (uint32_t *)(sm + 65536 + 64);
  volatile int *abort = (volatile int *)(sm + 65536 + 128);
  const int tid = threadIdx.x, warp = tid >> 5;
  const bool bf16 = P.mode == 2;
  const int rowb = bf16 ? 64 : 128;
  if (tid == 0) {
    mbar_init(&bars[0], 1);  // TMA
    mbar_init(&bars[1], 1);  // MMA done
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 4) {
    tmem_alloc(tbase, 256);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tbase;
  // A: thread r writes row r
  if (tid < 128) {
    const int r = tid;
    for (int c = 0; c < (bf16 ? 4 : 8); ++c) {
      uint32_t hi[4], lo[4];
      if (bf16) {
        for (int e = 0; e < 4; ++e) {
          float y0 = P.A[r * 32 + 8 * c + 2 * e], y1 = P.A[r * 32 + 8 * c + 2 * e + 1];
          __nv_bfloat162 h = __floats2bfloat162_rn(y0, y1);
          float2 hf = __bfloat1622float2(h);
          __nv_bfloat162 l = __floats2bfloat162_rn(y0 - hf.x, y1 - hf.y);
          hi[e] = *reinterpret_cast<uint32_t *>(&h);
          lo[e] = *reinterpret_cast<uint32_t *>(&l);
        }
        uint32_t off = (r >> 3) * 512 + (r & 7) * 64 + ((c ^ ((r & 7) >> 1)) << 4);
        *reinterpret_cast<uint4 *>(A0 + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4 *>(A1 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      } else {
        for (int e = 0; e < 4; ++e) {
          uint32_t t;
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(P.A[r * 32 + 4 * c + e]));
          hi[e] = t;
        }
        uint32_t off = (r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4);
        *reinterpret_cast<uint4 *>(A0 + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      }
    }
    fence_proxy_async_smem();
  }
  __syncthreads();
  if (tid == 128) {
    const int nbox = (P.N + 63) / 64;
    const uint32_t box_bytes = 64 * rowb;
    mbar_arrive_expect_tx(&bars[0], nbox * box_bytes * (bf16 ? 2 : 1));
    for (int i = 0; i < nbox; ++i) {
      tma_load_2d(B0 + i * box_bytes, &P.tm_b[0], 0, P.b_row_off + 64 * i, &bars[0]);
      if (bf16) tma_load_2d(B1 + i * box_bytes, &P.tm_b[1], 0, P.b_row_off + 64 * i, &bars[0]);
    }
    bool ok = mbar_wait(&bars[0], 0, abort);
    if (ok) {
      tc_fence_after();
      const uint32_t sbo = bf16 ? 512 : 1024, lay = bf16 ? 4 : 2;
      const uint32_t idesc = bf16 ? instr_desc(1, 1, 128, P.N) : instr_desc(2, 2, 128, P.N);
      const int nk = bf16 ? 2 : 4;
      uint32_t acc = 0;
      for (int ks = 0; ks < nk; ++ks) {
        uint64_t a0 = smem_desc(smem_u32(A0) + 32 * ks, sbo, lay);
        uint64_t b0 = smem_desc(smem_u32(B0) + 32 * ks, sbo, lay);
        if (bf16) {
          uint64_t a1 = smem_desc(smem_u32(A1) + 32 * ks, sbo, lay);
          uint64_t b1 = smem_desc(smem_u32(B1) + 32 * ks, sbo, lay);
          mma_f16(tmem + P.d_col_off, a0, b0, idesc, acc);
          acc = 1;
          mma_f16(tmem + P.d_col_off, a0, b1, idesc, 1);
          mma_f16(tmem + P.d_col_off, a1, b0, idesc, 1);
        } else {
          mma_tf32(tmem + P.d_col_off, a0, b0, idesc, acc);
          acc = 1;
        }
      }
      mma_commit(&bars[1]);
    } else {
      atomicExch(P.status, 1);
      *abort = 1;
    }
  }
  if (tid < 128) {
    if (mbar_wait(&bars[1], 0, abort)) {
      tc_fence_after();
      const int w = warp;
      for (int c0 = 0; c0 < P.N; c0 += 32) {
        uint32_t v[32];
        tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * w) << 16) + P.d_col_off + c0, v);
        tmem_wait_ld();
        const int r = tid;
        for (int j = 0; j < 32; ++j)
          if (c0 + j < P.N) P.D[r * P.N + c0 + j] = __uint_as_float(v[j]);
      }
    } else {
      atomicExch(P.status, 2);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                            CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn get_encode() {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return (EncodeFn)fn;
}

}  // namespace

// B is rows x 32 row-major floats (rows >= b_row_off + N).  Returns 0 on success.
extern "C" int umma_unit(int mode, int N, int rows, const float *A, const float *B, float *D,
                         int b_row_off, int d_col_off) {
  EncodeFn enc = get_encode();
  if (!enc) return 10;
  const bool bf16 = mode == 2;
  float *dA, *dD;
  void *dB[2] = {nullptr, nullptr};
  int *dst;
  cudaMalloc(&dA, 128 * 32 * 4);
  cudaMalloc(&dD, 128 * N * 4);
  cudaMalloc(&dst, 4);
  cudaMemset(dst, 0, 4);
  cudaMemcpy(dA, A, 128 * 32 * 4, cudaMemcpyHostToDevice);
  Params P{};
  if (bf16) {
    __nv_bfloat16 *h = new __nv_bfloat16[rows * 32], *l = new __nv_bfloat16[rows * 32];
    for (int i = 0; i < rows * 32; ++i) {
      h[i] = __float2bfloat16_rn(B[i]);
      l[i] = __float2bfloat16_rn(B[i] - __bfloat162float(h[i]));
    }
    for (int p = 0; p < 2; ++p) {
      cudaMalloc(&dB[p], rows * 32 * 2);
      cudaMemcpy(dB[p], p ? l : h, rows * 32 * 2, cudaMemcpyHostToDevice);
    }
    delete[] h;
    delete[] l;
  } else {
    float *t = new float[rows * 32];
    for (int i = 0; i < rows * 32; ++i) {
      uint32_t u;
      memcpy(&u, &B[i], 4);
      u = (u + 0x1000u) & 0xFFFFE000u;  // round to TF32 (ties away, as cvt.rna)
      memcpy(&t[i], &u, 4);
    }
    cudaMalloc(&dB[0], rows * 32 * 4);
    cudaMemcpy(dB[0], t, rows * 32 * 4, cudaMemcpyHostToDevice);
    delete[] t;
  }
  for (int p = 0; p < (bf16 ? 2 : 1); ++p) {
    cuuint64_t dims[2] = {32, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)32 * (bf16 ? 2 : 4)};
    cuuint32_t box[2] = {32, 64};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(&P.tm_b[p], bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                     dB[p], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     bf16 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return 11;
  }
  P.A = dA;
  P.D = dD;
  P.N = N;
  P.b_row_off = b_row_off;
  P.d_col_off = d_col_off;
  P.mode = mode;
  P.status = dst;
  cudaFuncSetAttribute(k_umma_unit, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem + 1024);
  k_umma_unit<<<1, 160, kSmem + 1024>>>(P);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    fprintf(stderr, "umma_unit: %s\n", cudaGetErrorString(e));
    return 12;
  }
  int st = 0;
  cudaMemcpy(&st, dst, 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(D, dD, 128 * N * 4, cudaMemcpyDeviceToHost);
  cudaFree(dA);
  cudaFree(dD);
  cudaFree(dst);
  for (void *p : dB)
    if (p) cudaFree(p);
  return st ? 20 + st : 0;
}

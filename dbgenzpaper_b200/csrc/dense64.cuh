// dense64.cuh -- FP64 dense kernels of the gradient path, written for this
// library: a tiled GEMM that skips the zero blocks of triangular operands
// and writes only the triangle its caller needs, with split-K partial tiles
// summed in a fixed order, and the inverse of an upper-triangular matrix.
//
//   gemm64:   C = op(A) op(B)  (+ C when accumulate), column-major
//             operands; per 64 x 64 output tile the k range is cut to
//             where the operands' triangles can be nonzero, and tiles
//             outside the requested output triangle are not launched.
//   trinv64:  X = U^-1 for U upper triangular (d x d, column-major).
//
// Used by the Cholesky adjoint (chol_adjoint.cu: U Ubar', U^-1 (.) U^-T,
// U'U) and by the FP64 factor gradient dU[l, t] = sum_n y[l][n] (p sbar)[t][n]
// (grad.cu).  No library GEMM: the same operand sizes run on CUDA cores in
// FP64 (the B200's FP64 rate is the same on CUDA cores and tensor cores).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace dense64 {
namespace {  // internal linkage: every translation unit that includes this gets its own copy

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

enum OutMode {
  kOutFull = 0,         // every C entry
  kOutLowerPhi = 1,     // i > j: v; i == j: v / 2; i < j: 0 (the Phi of the Cholesky adjoint)
  kOutStrictUpper = 2,  // i < j only (other entries untouched)
};

struct GemmArgs {
  int64_t m = 0, n = 0, k = 0;
  const double *A = nullptr;
  int64_t lda = 0;
  const double *B = nullptr;
  int64_t ldb = 0;
  double *C = nullptr;
  int64_t ldc = 0;
  // k range per output tile [i0, i1) x [j0, j1): from max(i0 if kmin_row,
  // j0 if kmin_col) to min(i1 if kmax_row, j1 if kmax_col, k)
  int kmin_row = 0, kmin_col = 0, kmax_row = 0, kmax_col = 0;
  int out = kOutFull;
  int accumulate = 0;  // C += product (else C = product)
  // split-K: splits > 1 writes partial tiles [split][tile_i][tile_j][64 x 64]
  // to `partial`, summed by k_gemm64_reduce
  int splits = 1;
  double *partial = nullptr;
};

__device__ __forceinline__ bool tile_needed(const GemmArgs &g, int64_t i0, int64_t i1, int64_t j0, int64_t j1) {
  if (g.out == kOutLowerPhi) return i1 - 1 >= j0;      // some i >= j
  if (g.out == kOutStrictUpper) return i0 < j1 - 1;    // some i < j
  return true;
}

__device__ __forceinline__ void tile_krange(const GemmArgs &g, int64_t i0, int64_t i1, int64_t j0, int64_t j1,
                                            int64_t &k0, int64_t &k1) {
  k0 = 0;
  if (g.kmin_row && i0 > k0) k0 = i0;
  if (g.kmin_col && j0 > k0) k0 = j0;
  k1 = g.k;
  if (g.kmax_row && i1 < k1) k1 = i1;
  if (g.kmax_col && j1 < k1) k1 = j1;
}

__device__ __forceinline__ double out_value(int out, int64_t i, int64_t j, double v, bool &write) {
  write = true;
  if (out == kOutLowerPhi) return i > j ? v : (i == j ? 0.5 * v : 0.0);
  if (out == kOutStrictUpper) write = i < j;
  return v;
}

// One 64 x 64 output tile per CTA (256 threads, 4 x 4 per thread: rows
// tx + 16 a, columns ty + 16 b), k in steps of 16 through shared memory, the
// next step's operands loaded into registers while this one is used.
// TA / TB: op(A) = A' / op(B) = B'.
template <bool TA, bool TB>
__global__ void __launch_bounds__(NT) k_gemm64(const GemmArgs g) {
  __shared__ double As[BK][BM + 1];
  __shared__ double Bs[BK][BN + 1];
  const int64_t tiles_n = (g.n + BN - 1) / BN;
  const int64_t ti = blockIdx.x / tiles_n, tj = blockIdx.x % tiles_n;
  const int64_t i0 = ti * BM, j0 = tj * BN;
  const int64_t i1 = i0 + BM < g.m ? i0 + BM : g.m, j1 = j0 + BN < g.n ? j0 + BN : g.n;
  if (!tile_needed(g, i0, i1, j0, j1)) return;
  int64_t k0, k1;
  tile_krange(g, i0, i1, j0, j1, k0, k1);
  // this split's share of the k range, in whole steps
  if (g.splits > 1) {
    const int64_t steps = (k1 > k0 ? k1 - k0 + BK - 1 : 0) / BK;
    const int64_t per = (steps + g.splits - 1) / g.splits;
    const int64_t s0 = k0 + (int64_t)blockIdx.y * per * BK;
    const int64_t s1 = s0 + per * BK;
    k1 = s1 < k1 ? s1 : k1;
    k0 = s0;
  }
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

  // operand loads: 1024 elements per tile, 4 per thread
  double ra[4], rb[4];
  auto load = [&](int64_t kk) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + NT * q;
      // A tile element (i, k): op N -> i fastest (coalesced), op T -> k fastest
      const int ai = TA ? e / BK : e % BM, ak = TA ? e % BK : e / BM;
      const int64_t gi = i0 + ai, gk = kk + ak;
      ra[q] = (gi < i1 && gk < k1) ? (TA ? g.A[gk + gi * g.lda] : g.A[gi + gk * g.lda]) : 0.0;
      // B tile element (k, j): op N -> k fastest, op T -> j fastest
      const int bj = TB ? e % BN : e / BK, bk = TB ? e / BN : e % BK;
      const int64_t gj = j0 + bj, gk2 = kk + bk;
      rb[q] = (gj < j1 && gk2 < k1) ? (TB ? g.B[gj + gk2 * g.ldb] : g.B[gk2 + gj * g.ldb]) : 0.0;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = tid + NT * q;
      const int ai = TA ? e / BK : e % BM, ak = TA ? e % BK : e / BM;
      As[ak][ai] = ra[q];
      const int bj = TB ? e % BN : e / BK, bk = TB ? e / BN : e % BK;
      Bs[bk][bj] = rb[q];
    }
  };
  if (k0 < k1) load(k0);
  for (int64_t kk = k0; kk < k1; kk += BK) {
    __syncthreads();
    store();
    __syncthreads();
    if (kk + BK < k1) load(kk + BK);
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[k][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[k][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
    }
  }
  if (g.splits > 1) {
    double *pt = g.partial + (((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * BM) * BN;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) pt[(ty + 16 * b) * BM + tx + 16 * a] = acc[a][b];
    return;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t i = i0 + tx + 16 * a, j = j0 + ty + 16 * b;
      if (i >= i1 || j >= j1) continue;
      bool w;
      double v = acc[a][b];
      if (g.accumulate) v += g.C[i + j * g.ldc];
      v = out_value(g.out, i, j, v, w);
      if (w) g.C[i + j * g.ldc] = v;
    }
}

// Sum of the split partial tiles in split order, then the output rule.
__global__ void k_gemm64_reduce(const GemmArgs g, int64_t n_tiles) {
  const int64_t tiles_n = (g.n + BN - 1) / BN;
  const int64_t tile = blockIdx.x;
  const int64_t ti = tile / tiles_n, tj = tile % tiles_n;
  const int64_t i0 = ti * BM, j0 = tj * BN;
  const int64_t i1 = i0 + BM < g.m ? i0 + BM : g.m, j1 = j0 + BN < g.n ? j0 + BN : g.n;
  if (!tile_needed(g, i0, i1, j0, j1)) return;
  for (int e = threadIdx.x; e < BM * BN; e += blockDim.x) {
    const int li = e % BM, lj = e / BM;
    const int64_t i = i0 + li, j = j0 + lj;
    if (i >= i1 || j >= j1) continue;
    double v = 0.0;
    for (int s = 0; s < g.splits; ++s) v += g.partial[((int64_t)s * n_tiles + tile) * BM * BN + e];
    bool w;
    if (g.accumulate) v += g.C[i + j * g.ldc];
    v = out_value(g.out, i, j, v, w);
    if (w) g.C[i + j * g.ldc] = v;
  }
}

// Bytes of partial tiles a split-K launch needs.
inline size_t gemm64_partial_bytes(const GemmArgs &g) {
  if (g.splits <= 1) return 0;
  const int64_t tiles = ((g.m + BM - 1) / BM) * ((g.n + BN - 1) / BN);
  return sizeof(double) * (size_t)g.splits * (size_t)tiles * BM * BN;
}

// Enqueues C = op(A) op(B) on `st` (one launch, or two with split-K).
// Returns the CUDA error of the launches.
template <bool TA, bool TB>
inline cudaError_t gemm64(const GemmArgs &g, cudaStream_t st, int *launches = nullptr) {
  if (g.m <= 0 || g.n <= 0) return cudaSuccess;
  const int64_t tiles = ((g.m + BM - 1) / BM) * ((g.n + BN - 1) / BN);
  k_gemm64<TA, TB><<<dim3((unsigned)tiles, (unsigned)(g.splits > 1 ? g.splits : 1)), NT, 0, st>>>(g);
  if (launches) ++*launches;
  if (g.splits > 1) {
    k_gemm64_reduce<<<(unsigned)tiles, 256, 0, st>>>(g, tiles);
    if (launches) ++*launches;
  }
  return cudaGetLastError();
}

// X = U^-1, U upper triangular (column-major, ld d; the strict lower
// triangle of U is not read), X upper triangular with zeros below the
// diagonal.  One CTA per column c: back substitution of U x = e_c from
// row c upwards, right-looking (after x_r is known, column r of U -- a
// contiguous read -- updates the rows above it); the right-hand side lives
// in shared memory (8 d bytes).
__global__ void k_trinv64(const double *U, int64_t d, double *X) {
  extern __shared__ double rhs[];
  const int64_t c = blockIdx.x;
  for (int64_t i = threadIdx.x; i < d; i += blockDim.x) rhs[i] = i == c ? 1.0 : 0.0;
  __syncthreads();
  for (int64_t r = c; r >= 0; --r) {
    const double xr = rhs[r] / U[r * d + r];
    const double *ur = U + r * d;
    for (int64_t i = threadIdx.x; i < r; i += blockDim.x) rhs[i] = fma(-ur[i], xr, rhs[i]);
    if (threadIdx.x == 0) X[c * d + r] = xr;
    __syncthreads();
  }
  for (int64_t i = c + 1 + threadIdx.x; i < d; i += blockDim.x) X[c * d + i] = 0.0;
}

// The same back substitution with the next column of U loaded into
// registers while the current one is applied, and one barrier per step:
// every thread forms x_r itself (the same operation on the same operands),
// so the step's only exchange is the right-hand side in shared memory.
// Thread t owns rows t + 128 q, q < Q (d <= 128 Q).
template <int Q>
__global__ void __launch_bounds__(128) k_trinv64_pf(const double *U, int64_t d, double *X) {
  extern __shared__ double rhs[];
  const int64_t c = blockIdx.x;
  const int tid = threadIdx.x;
  for (int64_t i = tid; i < d; i += 128) rhs[i] = i == c ? 1.0 : 0.0;
  double ucur[Q], unext[Q];
  // x_r = rhs_r * (1 / U_rr): the reciprocal of the next step's diagonal is
  // formed while the current step runs, so the chain of steps carries a
  // multiplication, not a division (within an ulp of rhs_r / U_rr)
  double dcur = 1.0 / U[c * d + c], dnext = 1.0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int64_t i = tid + 128 * q;
    ucur[q] = i < c ? U[c * d + i] : 0.0;
  }
  __syncthreads();
  for (int64_t r = c; r >= 0; --r) {
    if (r > 0) {
      const double *un = U + (r - 1) * d;
      dnext = 1.0 / un[r - 1];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int64_t i = tid + 128 * q;
        unext[q] = i < r - 1 ? un[i] : 0.0;
      }
    }
    const double xr = rhs[r] * dcur;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int64_t i = tid + 128 * q;
      if (i < r) rhs[i] = fma(-ucur[q], xr, rhs[i]);
    }
    if (tid == 0) X[c * d + r] = xr;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) ucur[q] = unext[q];
    dcur = dnext;
  }
  for (int64_t i = c + 1 + tid; i < d; i += 128) X[c * d + i] = 0.0;
}

inline size_t trinv64_smem(int64_t d) { return sizeof(double) * (size_t)d; }

template <typename K>
inline cudaError_t trinv64_launch(K kern, const double *U, int64_t d, double *X, cudaStream_t st) {
  const size_t smem = trinv64_smem(d);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<(unsigned)d, 128, smem, st>>>(U, d, X);
  return cudaGetLastError();
}

inline cudaError_t trinv64(const double *U, int64_t d, double *X, cudaStream_t st, int *launches = nullptr) {
  if (launches) ++*launches;
  if (d <= 128 * 2) return trinv64_launch(k_trinv64_pf<2>, U, d, X, st);
  if (d <= 128 * 4) return trinv64_launch(k_trinv64_pf<4>, U, d, X, st);
  if (d <= 128 * 8) return trinv64_launch(k_trinv64_pf<8>, U, d, X, st);
  if (d <= 128 * 16) return trinv64_launch(k_trinv64_pf<16>, U, d, X, st);
  return trinv64_launch(k_trinv64, U, d, X, st);
}

}  // namespace
}  // namespace dense64

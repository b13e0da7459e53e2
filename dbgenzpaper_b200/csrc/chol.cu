// chol.cu -- FP64 blocked Cholesky factorisations on the GPU.
//
//  * cholesky_genz!  (reference src/cholesky.jl:445-628): Genz variable
//    reordering inside every bs2 panel, panel-restricted argmin pivoting,
//    s_vec carried only inside the current panel.
//  * cholesky_classic! (src/cholesky.jl:144-242): no pivoting.
//
// Arithmetic contract: every sum the reference hands to BLAS (mul!, ldiv!,
// dot) is evaluated here as ONE fused-multiply-add chain in ascending index
// order, and every other operation is a single IEEE operation with
// contraction disabled (dm_* in detmath.h).  The CPU checker follows the
// same contract, so U, the pivot permutation and the permuted bounds agree
// bit for bit.  Parallelism comes from computing independent chains
// concurrently (one chain per output element), never from splitting a
// chain.
//
// Layout: M is d x d column-major in HBM (8 MB at d = 1000, L2 resident);
// a sequential pivot step runs in one CTA (latency-bound: scores, argmin,
// swaps, row update), the trailing Schur updates and triangular solves run
// on the whole GPU.
#include "internal.cuh"
#include "detmath.h"
#include "chol_dev.cuh"
#include <cfloat>

namespace {

constexpr int kStepThreads = 1024;

__global__ void k_diag_absmax(const double *M, int64_t n, double *out) {
  __shared__ double sh[32];
  double mx = 0.0;
  bool nan = false;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    double v = fabs(M[j * n + j]);
    if (v != v) nan = true;
    else if (v > mx) mx = v;
  }
  nan = __syncthreads_or(nan);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
    out[0] = nan ? NAN : dm_mul(DBL_EPSILON, r);
  }
}

__global__ void k_scale_vec(const double *M, int64_t n, double *scale) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double v = M[j * n + j];
  scale[j] = v > 0 ? dm_sqrt(v) : 1.0;
}

// src/cholesky.jl:458-473 (genz, mirror = 1) / :154-166 (classic, mirror = 0)
__global__ void k_scale_apply(double *M, int64_t n, double *a, double *b, const double *scale,
                              int mirror) {
  int64_t j = blockIdx.y;
  double s_j = scale[j];
  double inv_s_j = dm_div(1.0, s_j);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= j;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i == j) {
      M[j * n + j] = 1.0;
      a[j] = dm_mul(a[j], inv_s_j);
      b[j] = dm_mul(b[j], inv_s_j);
    } else {
      double val = dm_mul(M[j * n + i], dm_div(inv_s_j, scale[i]));
      M[j * n + i] = val;
      if (mirror) M[i * n + j] = val;
    }
  }
}

// One bs1 block of cholesky_genz! (src/cholesky.jl:494-572), one CTA.
__global__ void __launch_bounds__(kStepThreads)
k_genz_block(double *M, int64_t n, double *a, double *b, double *dvec, double *svec, double *ovec, int64_t *perm,
             int64_t i0, int64_t i1, int64_t ii1, const double *eps0_ptr, int64_t *rank) {
  cholk::genz_block_dev(M, n, a, b, dvec, svec, ovec, perm, i0, i1, ii1, eps0_ptr, rank);
}
// The same with the panel's vectors in shared memory (panels of up to
// kGenzSmemPanel candidates).
constexpr int64_t kGenzSmemPanel = 1024;
__global__ void __launch_bounds__(kStepThreads)
k_genz_block_smem(double *M, int64_t n, double *a, double *b, double *dvec, double *svec, int64_t *perm, int64_t i0,
                  int64_t i1, int64_t ii1, const double *eps0_ptr, int64_t *rank) {
  extern __shared__ double genz_sh[];
  cholk::genz_block_smem(M, n, a, b, dvec, svec, perm, i0, i1, ii1, eps0_ptr, rank, genz_sh);
}

// The same with the block's factor entries on chip (panels of up to
// cholk::kOnchipSlots candidates, blocks of up to cholk::kOnchipPiv pivots):
// the slot warps and the y_i warp.
constexpr int kOnchipThreads = cholk::kOnchipSlots + 32;
__global__ void __launch_bounds__(kOnchipThreads)
k_genz_block_onchip(double *M, int64_t n, double *a, double *b, double *dvec, double *svec, int64_t *perm,
                    int64_t i0, int64_t i1, int64_t ii1, const double *eps0_ptr, int64_t *rank) {
  extern __shared__ double genz_sh[];
  cholk::genz_block_onchip(M, n, a, b, dvec, svec, perm, i0, i1, ii1, eps0_ptr, rank, genz_sh);
}

// One bs1 block of cholesky_rowmax! (src/cholesky.jl:290-357), one CTA: the
// pivot is the largest remaining diagonal of the panel (first on ties, NaN
// never chosen unless it is the current row's own), the rank test m_ii > 0
// comes before the swap, a and b are not swapped.  The same operations in
// the same order as the checker's restatement.
__global__ void __launch_bounds__(kStepThreads)
k_rowmax_block(double *M, int64_t n, double *dvec, int64_t *perm, int64_t i0, int64_t i1, int64_t ii1,
               int64_t *rank) {
  __shared__ double red_v[32];
  __shared__ int64_t red_i[32];
  __shared__ int64_t sh_im;
  __shared__ double sh_mii;
  __shared__ int sh_stop;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (rank[0] < n) return;
  for (int64_t k = i0 + tid; k <= ii1; k += blockDim.x) dvec[k] = 0.0;
  __syncthreads();
  // larger wins; equal values keep the smaller index; NaN (INT64_MAX index) never wins
  auto better = [](double v2, int64_t i2, double v, int64_t i) {
    if (i2 == INT64_MAX) return false;
    if (i == INT64_MAX) return true;
    return v2 > v || (v2 == v && i2 < i);
  };
  for (int64_t i = i0; i <= i1; ++i) {
    double bv = 0.0;
    int64_t bi = INT64_MAX;
    for (int64_t k = i + tid; k <= ii1; k += blockDim.x) {
      const double v = dm_sub(M[k * n + k], dvec[k]);
      if (v == v && better(v, k, bv, bi)) { bv = v; bi = k; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double v2 = __shfl_down_sync(0xffffffffu, bv, off);
      const int64_t i2 = __shfl_down_sync(0xffffffffu, bi, off);
      if (lane + off < 32 && better(v2, i2, bv, bi)) { bv = v2; bi = i2; }
    }
    if (lane == 0) { red_v[wid] = bv; red_i[wid] = bi; }
    __syncthreads();
    if (tid == 0) {
      double v = red_v[0];
      int64_t im = red_i[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
        if (better(red_v[w], red_i[w], v, im)) { v = red_v[w]; im = red_i[w]; }
      const double m_own = dm_sub(M[i * n + i], dvec[i]);
      if (m_own != m_own || im == INT64_MAX) im = i;  // the scan starts from row i's own value
      double m_ii = dm_sub(M[im * n + im], dvec[im]);
      int stop = 0;
      if (m_ii > 0) {
        m_ii = dm_sqrt(m_ii);
      } else {
        rank[0] = i;  // 0-based i == the reference's i - 1
        stop = 1;
      }
      if (!stop && im != i) {
        const int64_t tp = perm[i]; perm[i] = perm[im]; perm[im] = tp;
        const double t = dvec[im]; dvec[im] = dvec[i]; dvec[i] = t;
      }
      sh_im = im;
      sh_mii = m_ii;
      sh_stop = stop;
    }
    __syncthreads();
    if (sh_stop) return;
    const int64_t im = sh_im;
    if (im != i) {  // rows over columns i0..n, then full columns
      for (int64_t k = i0 + tid; k < n; k += blockDim.x) {
        const double t = M[k * n + i];
        M[k * n + i] = M[k * n + im];
        M[k * n + im] = t;
      }
      __syncthreads();
      for (int64_t k = tid; k < n; k += blockDim.x) {
        const double t = M[i * n + k];
        M[i * n + k] = M[im * n + k];
        M[im * n + k] = t;
      }
      __syncthreads();
    }
    const double m_ii = sh_mii;
    if (tid == 0) M[i * n + i] = m_ii;
    if (i == i0) {
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        const double m_ij = dm_div(M[j * n + i], m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        dvec[j] = dm_add(dvec[j], dm_mul(m_ij, m_ij));
      }
    } else if (i < ii1) {
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        double acc = 0.0;
        for (int64_t l = i0; l <= i - 1; ++l) acc = dm_fma(M[l * n + j], M[i * n + l], acc);
        const double m_ij = dm_div(dm_sub(M[i * n + j], acc), m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        dvec[j] = dm_add(dvec[j], dm_mul(m_ij, m_ij));
      }
    }
    __syncthreads();
  }
}

// C[j,k] -= sum_{l=p0..p1} A(l,j) B(l,k) over [c0, c1]^2, one tile per CTA.
constexpr int kTile = cholk::kTile;
__global__ void __launch_bounds__(256)
k_schur_update(double *M, int64_t n, int64_t p0, int64_t p1, int64_t c0, int64_t c1, int a_row,
               const int64_t *rank) {
  // after a rank failure the reference stops (src/cholesky.jl:575-576, 586-587, ...): no update
  if (rank && rank[0] < n) return;
  cholk::schur_tile_dev(M, n, p0, p1, c0, c1, a_row, c0 + blockIdx.x * (int64_t)kTile,
                        c0 + blockIdx.y * (int64_t)kTile);
}

// ldiv!(UpperTriangular(M[p0:p1,p0:p1])', M[p0:p1, c0:c1]): forward
// substitution X[r] = (X[r] - sum_{l<r} U[l,r] X[l]) / U[r,r] per column.
//
// Right-looking wavefront with the same arithmetic as the left-looking
// form: row r's accumulator receives fma(U[l,r], X[l], acc) for l = p0,
// p0+1, ..., r-1 in that order, starting from 0, so every X[r] is the same
// ascending fma chain.  One warp per column c; lane i owns rows
// q0 + i + 32k (k < kTrsmSlots) of a pass of kTrsmPass rows; the owner of
// row l finishes X[l] and broadcasts it, then every lane updates its rows
// r > l.  U[l0:l0+31, pass rows] is staged in shared memory (coalesced
// 256-byte row segments of the column-major M) and shared by the CTA's
// kTrsmWarps columns; the chunks are double-buffered, the next one copied by
// cp.async while the current one is used (U is read only: X's columns lie
// beyond p1).
constexpr int kTrsmWarps = 8, kTrsmSlots = 8, kTrsmPass = 32 * kTrsmSlots, kTrsmLc = 32;
constexpr int kTrsmLd = kTrsmPass + 1;  // padded row of the staged chunk
constexpr int kTrsmChunk = kTrsmLc * kTrsmLd;  // doubles per staged chunk
__device__ __forceinline__ void trsm_cp8(double *dst, const double *src, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__global__ void __launch_bounds__(32 * kTrsmWarps)
k_trsm_ut(double *M, int64_t n, int64_t p0, int64_t p1, int64_t c0, int64_t c1, const int64_t *rank) {
  if (rank && rank[0] < n) return;  // after a rank failure: no update
  // two chunks [kTrsmLc][kTrsmLd]: Us[lc * kTrsmLd + rr] = U[l0 + lc, q0 + rr]
  extern __shared__ double Us2[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t c = c0 + (int64_t)blockIdx.x * kTrsmWarps + warp;
  const bool active = c <= c1;
  double *X = M + (active ? c : c0) * n;
  // the chunk sequence: passes q0, and in each the chunks l0 = p0, p0 + 32, ... <= q1
  auto stage = [&](int buf, int64_t q0, int64_t l0) {
    const int64_t q1 = q0 + kTrsmPass - 1 < p1 ? q0 + kTrsmPass - 1 : p1;
    const int nrows = (int)(q1 - q0 + 1);
    const int nl = (int)((q1 - l0 + 1) < kTrsmLc ? (q1 - l0 + 1) : kTrsmLc);
    double *Us = Us2 + buf * kTrsmChunk;
    for (int idx = threadIdx.x; idx < kTrsmPass * kTrsmLc; idx += blockDim.x) {
      const int rr = idx / kTrsmLc, lc = idx % kTrsmLc;
      const bool v = rr < nrows && lc < nl;
      trsm_cp8(Us + lc * kTrsmLd + rr, v ? M + (q0 + rr) * n + l0 + lc : M, v);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto next_chunk = [&](int64_t &q0, int64_t &l0) -> bool {  // advance; false at the end
    const int64_t q1 = q0 + kTrsmPass - 1 < p1 ? q0 + kTrsmPass - 1 : p1;
    l0 += kTrsmLc;
    if (l0 > q1) {
      q0 += kTrsmPass;
      l0 = p0;
    }
    return q0 <= p1;
  };
  int64_t sq = p0, sl = p0;  // the chunk being staged
  bool more = true;
  stage(0, sq, sl);
  int buf = 0;
  for (int64_t q0 = p0; q0 <= p1; q0 += kTrsmPass) {
    const int64_t q1 = q0 + kTrsmPass - 1 < p1 ? q0 + kTrsmPass - 1 : p1;
    const int nrows = (int)(q1 - q0 + 1);
    double acc[kTrsmSlots], xin[kTrsmSlots];
#pragma unroll
    for (int k = 0; k < kTrsmSlots; ++k) {
      acc[k] = 0.0;
      const int rr = lane + 32 * k;
      xin[k] = (active && rr < nrows) ? X[q0 + rr] : 0.0;
    }
    for (int64_t l0 = p0; l0 <= q1; l0 += kTrsmLc) {
      const int nl = (int)((q1 - l0 + 1) < kTrsmLc ? (q1 - l0 + 1) : kTrsmLc);
      // the next chunk into the other buffer (the buffer it overwrites was
      // last read before the barrier that ended the previous chunk)
      __syncthreads();
      if (more) more = next_chunk(sq, sl);
      if (more) {
        stage(buf ^ 1, sq, sl);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
      __syncthreads();
      const double *Us = Us2 + buf * kTrsmChunk;
      buf ^= 1;
      if (!active) continue;
      if (l0 < q0) {
        // rows of earlier passes: X[l] is final (written by this lane)
        const double xl = lane < nl ? X[l0 + lane] : 0.0;
        for (int lc = 0; lc < nl; ++lc) {
          const double xv = __shfl_sync(0xffffffffu, xl, lc);
          const double *u = Us + lc * kTrsmLd;
#pragma unroll
          for (int k = 0; k < kTrsmSlots; ++k) {
            const int rr = lane + 32 * k;
            if (rr < nrows) acc[k] = dm_fma(u[rr], xv, acc[k]);
          }
        }
      } else {
        // rows of this pass: slot ks holds rows l0 .. l0+31, lane lc owns l0+lc
        const int ks = (int)((l0 - q0) / 32);
        for (int lc = 0; lc < nl; ++lc) {
          double mine = 0.0;
#pragma unroll
          for (int k = 0; k < kTrsmSlots; ++k)
            if (k == ks && lane == lc) {
              xin[k] = dm_div(dm_sub(xin[k], acc[k]), Us[lc * kTrsmLd + (int)(l0 - q0) + lc]);
              mine = xin[k];
            }
          const double xv = __shfl_sync(0xffffffffu, mine, lc);
          const double *u = Us + lc * kTrsmLd;
          const int rl = (int)(l0 - q0) + lc;  // pass-local row of l
#pragma unroll
          for (int k = 0; k < kTrsmSlots; ++k) {
            const int rr = lane + 32 * k;
            if (rr > rl && rr < nrows) acc[k] = dm_fma(u[rr], xv, acc[k]);
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int k = 0; k < kTrsmSlots; ++k) {
        const int rr = lane + 32 * k;
        if (rr < nrows) X[q0 + rr] = xin[k];
      }
    }
    __syncwarp();
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// One bs1 block of cholesky_classic! (src/cholesky.jl:180-198), one CTA.
__global__ void __launch_bounds__(kStepThreads)
k_classic_block(double *M, int64_t n, int64_t i0, int64_t i1) {
  for (int64_t i = i0; i <= i1; ++i) {
    __shared__ double sh_mii;
    if (threadIdx.x == 0) {
      double m_ii = M[i * n + i];
      if (i > i0) {
        double acc = 0.0;
        for (int64_t l = i0; l <= i - 1; ++l) acc = dm_fma(M[i * n + l], M[i * n + l], acc);
        m_ii = dm_sub(m_ii, acc);
      }
      m_ii = dm_sqrt(m_ii);
      M[i * n + i] = m_ii;
      sh_mii = m_ii;
    }
    __syncthreads();
    const double m_ii = sh_mii;
    for (int64_t j = i + 1 + threadIdx.x; j <= i1; j += blockDim.x) {
      if (i > i0 && i < i1) {
        double acc = 0.0;
        for (int64_t l = i0; l <= i - 1; ++l) acc = dm_fma(M[j * n + l], M[i * n + l], acc);
        M[j * n + i] = dm_sub(M[j * n + i], acc);
        M[i * n + j] = 0.0;
      }
      M[j * n + i] = dm_div(M[j * n + i], m_ii);
    }
    __syncthreads();
  }
}

__global__ void k_truncate(double *U, int64_t nn, double min_val) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn;
       t += (int64_t)gridDim.x * blockDim.x)
    if (fabs(U[t]) < min_val) U[t] = 0.0;
}

__global__ void k_band(double *U, int64_t d, int64_t band) {
  const int64_t t = blockIdx.y;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < t - band; l += (int64_t)gridDim.x * blockDim.x)
    U[t * d + l] = 0.0;
}

// Ub[i + j d] = U[(d-1-j) + (d-1-i) d]: the anti-transpose (coefficients of
// the adjoint recurrence, policies.cuh)
__global__ void k_anti_transpose(const double *U, int64_t d, double *Ub) {
  const int64_t j = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < d; i += (int64_t)gridDim.x * blockDim.x)
    Ub[j * d + i] = U[(d - 1 - i) * d + (d - 1 - j)];
}

__global__ void k_targets(const double *U, int64_t n, const double *a, const double *b,
                          TargetParams64 *t64, TargetParams32 *t32) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double c2 = sqrt(2.0);
  double inv_u = 1.0 / (U[t * n + t] * c2);
  t64[t] = TargetParams64{a[t], b[t], inv_u};
  t32[t] = TargetParams32{(float)a[t], (float)b[t], (float)inv_u, 0.f};
}

__global__ void k_to_f32(const double *src, float *dst, int64_t nn) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn;
       t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = (float)src[t];
}

int launch_schur(dbgz_ctx *ctx, double *M, int64_t n, int64_t p0, int64_t p1, int64_t c0,
                 int64_t c1, int a_row, const int64_t *rank = nullptr) {
  if (c1 < c0 || p1 < p0) return DBGZ_OK;
  int64_t nt = (c1 - c0 + kTile) / kTile;
  dim3 grid((unsigned)nt, (unsigned)nt);
  k_schur_update<<<grid, 256, 0, ctx->stream>>>(M, n, p0, p1, c0, c1, a_row, rank);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int launch_trsm(dbgz_ctx *ctx, double *M, int64_t n, int64_t p0, int64_t p1, int64_t c0,
                int64_t c1, const int64_t *rank = nullptr) {
  if (c1 < c0) return DBGZ_OK;
  const int64_t nc = c1 - c0 + 1;
  const size_t smem = sizeof(double) * 2 * kTrsmChunk;
  // 132 KB of dynamic shared memory needs the opt-in, once per device
  static bool attr_set[64] = {};
  if (ctx->device < 0 || ctx->device >= 64 || !attr_set[ctx->device]) {
    DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(k_trsm_ut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (ctx->device >= 0 && ctx->device < 64) attr_set[ctx->device] = true;
  }
  k_trsm_ut<<<(unsigned)((nc + kTrsmWarps - 1) / kTrsmWarps), 32 * kTrsmWarps, smem, ctx->stream>>>(M, n, p0, p1,
                                                                                                    c0, c1, rank);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int scale_correlation(dbgz_ctx *ctx, double *M, int64_t n, double *a, double *b, double *scale,
                      int mirror) {
  k_scale_vec<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(M, n, scale);
  dbgz_count_launch(ctx);
  dim3 grid((unsigned)((n + 255) / 256), (unsigned)n);
  k_scale_apply<<<grid, 256, 0, ctx->stream>>>(M, n, a, b, scale, mirror);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

}  // namespace

int dbgz_chol_genz_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b, int64_t bs1,
                       int64_t bs2, int64_t bs3, int64_t bs4, int64_t *perm, double *scale,
                       int64_t *rank_host) {
  if (bs1 < 1 || bs2 < 1 || bs3 < 1 || bs4 < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "block sizes must be positive");
  DevBuf work;
  DBGZ_TRY(dbgz_ensure(ctx, work, sizeof(double) * (3 * n + 2) + sizeof(int64_t) * 2));
  double *dvec = (double *)work.p, *svec = dvec + n, *ovec = svec + n, *eps0 = ovec + n;
  int64_t *rank = (int64_t *)(eps0 + 2);
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(dvec, 0, sizeof(double) * 3 * n, st);
  k_diag_absmax<<<1, 1024, 0, st>>>(M, n, eps0);
  dbgz_count_launch(ctx);
  int st_ = scale_correlation(ctx, M, n, a, b, scale, 1);
  if (st_) { dbgz_release(work); return st_; }
  {
    std::vector<int64_t> id(n);
    for (int64_t i = 0; i < n; ++i) id[i] = i;
    cudaMemcpyAsync(perm, id.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
    int64_t rn = n;
    cudaMemcpyAsync(rank, &rn, sizeof(int64_t), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
  }
  int rc = DBGZ_OK;
  for (int64_t iv0 = 0; iv0 < n && rc == DBGZ_OK; iv0 += bs4) {
    int64_t iv1 = std::min(n - 1, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1 && rc == DBGZ_OK; iii0 += bs3) {
      int64_t iii1 = std::min(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1 && rc == DBGZ_OK; ii0 += bs2) {
        int64_t ii1 = std::min(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1 && rc == DBGZ_OK; i0 += bs1) {
          int64_t i1 = std::min(ii1, i0 + bs1 - 1);
          const int64_t panel = ii1 - i0 + 1;
          if (panel <= cholk::kOnchipSlots && i1 - i0 + 1 <= cholk::kOnchipPiv) {
            static bool attr_oc[64] = {};
            if (ctx->device < 0 || ctx->device >= 64 || !attr_oc[ctx->device]) {
              cudaFuncSetAttribute(k_genz_block_onchip, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)cholk::genz_block_onchip_bytes(cholk::kOnchipSlots));
              if (ctx->device >= 0 && ctx->device < 64) attr_oc[ctx->device] = true;
            }
            k_genz_block_onchip<<<1, kOnchipThreads, cholk::genz_block_onchip_bytes(panel), st>>>(
                M, n, a, b, dvec, svec, perm, i0, i1, ii1, eps0, rank);
          } else if (panel <= kGenzSmemPanel) {
            const size_t sm = cholk::genz_block_smem_bytes(panel);
            static bool attr[64] = {};
            if (ctx->device < 0 || ctx->device >= 64 || !attr[ctx->device]) {
              cudaFuncSetAttribute(k_genz_block_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)cholk::genz_block_smem_bytes(kGenzSmemPanel));
              if (ctx->device >= 0 && ctx->device < 64) attr[ctx->device] = true;
            }
            k_genz_block_smem<<<1, kStepThreads, sm, st>>>(M, n, a, b, dvec, svec, perm, i0, i1, ii1, eps0, rank);
          } else {
            k_genz_block<<<1, kStepThreads, 0, st>>>(M, n, a, b, dvec, svec, ovec, perm, i0, i1, ii1, eps0, rank);
          }
          dbgz_count_launch(ctx);
          if (i1 < ii1) rc = launch_schur(ctx, M, n, i0, i1, i1 + 1, ii1, 1, rank);
        }
        if (ii1 < iii1 && rc == DBGZ_OK) {
          rc = launch_trsm(ctx, M, n, ii0, ii1, ii1 + 1, iii1, rank);
          if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, ii0, ii1, ii1 + 1, iii1, 0, rank);
        }
      }
      if (iii1 < iv1 && rc == DBGZ_OK) {
        rc = launch_trsm(ctx, M, n, iii0, iii1, iii1 + 1, iv1, rank);
        if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, iii0, iii1, iii1 + 1, iv1, 0, rank);
      }
    }
    if (iv1 < n - 1 && rc == DBGZ_OK) {
      rc = launch_trsm(ctx, M, n, iv0, iv1, iv1 + 1, n - 1, rank);
      if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, iv0, iv1, iv1 + 1, n - 1, 0, rank);
    }
  }
  // Blocks after a rank failure return immediately (they read rank < n),
  // and the Schur updates after it only touch entries the reference leaves
  // as scratch beyond the failure point; callers reject rank < n anyway.
  if (rc == DBGZ_OK) {
    cudaError_t e = cudaMemcpyAsync(rank_host, rank, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_genz: %s", cudaGetErrorString(e));
  }
  cudaStreamSynchronize(st);
  dbgz_release(work);
  return rc;
}

// cholesky_rowmax! (src/cholesky.jl:244-432) on the device: the Genz
// driver's block structure with the diagonal-pivoting block step.
int dbgz_chol_rowmax_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b, int64_t bs1, int64_t bs2,
                         int64_t bs3, int64_t bs4, int64_t *perm, double *scale, int64_t *rank_host) {
  if (bs1 < 1 || bs2 < 1 || bs3 < 1 || bs4 < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "block sizes must be positive");
  DevBuf work;
  DBGZ_TRY(dbgz_ensure(ctx, work, sizeof(double) * (n + 1) + sizeof(int64_t) * 2));
  double *dvec = (double *)work.p;
  int64_t *rank = (int64_t *)(dvec + n + 1);
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(dvec, 0, sizeof(double) * n, st);
  int rc = scale_correlation(ctx, M, n, a, b, scale, 1);
  if (rc) {
    dbgz_release(work);
    return rc;
  }
  {
    std::vector<int64_t> id(n);
    for (int64_t i = 0; i < n; ++i) id[i] = i;
    cudaMemcpyAsync(perm, id.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
    int64_t rn = n;
    cudaMemcpyAsync(rank, &rn, sizeof(int64_t), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
  }
  for (int64_t iv0 = 0; iv0 < n && rc == DBGZ_OK; iv0 += bs4) {
    int64_t iv1 = std::min(n - 1, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1 && rc == DBGZ_OK; iii0 += bs3) {
      int64_t iii1 = std::min(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1 && rc == DBGZ_OK; ii0 += bs2) {
        int64_t ii1 = std::min(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1 && rc == DBGZ_OK; i0 += bs1) {
          int64_t i1 = std::min(ii1, i0 + bs1 - 1);
          k_rowmax_block<<<1, kStepThreads, 0, st>>>(M, n, dvec, perm, i0, i1, ii1, rank);
          dbgz_count_launch(ctx);
          if (i1 < ii1) rc = launch_schur(ctx, M, n, i0, i1, i1 + 1, ii1, 1, rank);
        }
        if (ii1 < iii1 && rc == DBGZ_OK) {
          rc = launch_trsm(ctx, M, n, ii0, ii1, ii1 + 1, iii1, rank);
          if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, ii0, ii1, ii1 + 1, iii1, 0, rank);
        }
      }
      if (iii1 < iv1 && rc == DBGZ_OK) {
        rc = launch_trsm(ctx, M, n, iii0, iii1, iii1 + 1, iv1, rank);
        if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, iii0, iii1, iii1 + 1, iv1, 0, rank);
      }
    }
    if (iv1 < n - 1 && rc == DBGZ_OK) {
      rc = launch_trsm(ctx, M, n, iv0, iv1, iv1 + 1, n - 1, rank);
      if (rc == DBGZ_OK) rc = launch_schur(ctx, M, n, iv0, iv1, iv1 + 1, n - 1, 0, rank);
    }
  }
  if (rc == DBGZ_OK) {
    cudaError_t e = cudaMemcpyAsync(rank_host, rank, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "cholesky_rowmax: %s", cudaGetErrorString(e));
  }
  cudaStreamSynchronize(st);
  dbgz_release(work);
  return rc;
}

int dbgz_chol_classic_dev(dbgz_ctx *ctx, int64_t n, double *M, double *a, double *b,
                          int64_t bs1, int64_t bs2, int64_t bs3, int64_t bs4, double *scale) {
  if (bs1 < 1 || bs2 < 1 || bs3 < 1 || bs4 < 1)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "block sizes must be positive");
  cudaStream_t st = ctx->stream;
  DBGZ_TRY(scale_correlation(ctx, M, n, a, b, scale, 0));
  for (int64_t iv0 = 0; iv0 < n; iv0 += bs4) {
    int64_t iv1 = std::min(n - 1, iv0 + bs4 - 1);
    for (int64_t iii0 = iv0; iii0 <= iv1; iii0 += bs3) {
      int64_t iii1 = std::min(iv1, iii0 + bs3 - 1);
      for (int64_t ii0 = iii0; ii0 <= iii1; ii0 += bs2) {
        int64_t ii1 = std::min(iii1, ii0 + bs2 - 1);
        for (int64_t i0 = ii0; i0 <= ii1; i0 += bs1) {
          int64_t i1 = std::min(ii1, i0 + bs1 - 1);
          k_classic_block<<<1, kStepThreads, 0, st>>>(M, n, i0, i1);
          dbgz_count_launch(ctx);
          if (i1 < ii1) {
            DBGZ_TRY(launch_trsm(ctx, M, n, i0, i1, i1 + 1, ii1));
            DBGZ_TRY(launch_schur(ctx, M, n, i0, i1, i1 + 1, ii1, 0));
          }
        }
        if (ii1 < iii1) {
          DBGZ_TRY(launch_trsm(ctx, M, n, ii0, ii1, ii1 + 1, iii1));
          DBGZ_TRY(launch_schur(ctx, M, n, ii0, ii1, ii1 + 1, iii1, 0));
        }
      }
      if (iii1 < iv1) {
        DBGZ_TRY(launch_trsm(ctx, M, n, iii0, iii1, iii1 + 1, iv1));
        DBGZ_TRY(launch_schur(ctx, M, n, iii0, iii1, iii1 + 1, iv1, 0));
      }
    }
    if (iv1 < n - 1) {
      DBGZ_TRY(launch_trsm(ctx, M, n, iv0, iv1, iv1 + 1, n - 1));
      DBGZ_TRY(launch_schur(ctx, M, n, iv0, iv1, iv1 + 1, n - 1, 0));
    }
  }
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return DBGZ_OK;
}

int dbgz_truncate_dev(dbgz_ctx *ctx, int64_t n, double *U, double eps_T) {
  double min_val = eps_T / (double)(n * 9);
  int64_t nn = n * n;
  int blocks = (int)std::min<int64_t>((nn + 255) / 256, 4096);
  k_truncate<<<blocks, 256, 0, ctx->stream>>>(U, nn, min_val);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_band_dev(dbgz_ctx *ctx, int64_t d, double *U, int64_t band) {
  dim3 g((unsigned)std::max<int64_t>(1, (d + 255) / 256), (unsigned)d);
  k_band<<<g, 256, 0, ctx->stream>>>(U, d, band);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_make_targets(dbgz_problem *p) {
  dbgz_ctx *ctx = p->ctx;
  int64_t n = p->d;
  DBGZ_TRY(dbgz_ensure(ctx, p->tgt64, sizeof(TargetParams64) * n));
  DBGZ_TRY(dbgz_ensure(ctx, p->tgt32, sizeof(TargetParams32) * n));
  k_targets<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
      (const double *)p->U.p, n, (const double *)p->a.p, (const double *)p->b.p,
      (TargetParams64 *)p->tgt64.p, (TargetParams32 *)p->tgt32.p);
  dbgz_count_launch(p->ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_make_U32(dbgz_problem *p) {
  dbgz_ctx *ctx = p->ctx;
  int64_t nn = p->d * p->d;
  DBGZ_TRY(dbgz_ensure(ctx, p->U32, sizeof(float) * nn));
  int blocks = (int)std::min<int64_t>((nn + 255) / 256, 4096);
  k_to_f32<<<blocks, 256, 0, ctx->stream>>>((const double *)p->U.p, (float *)p->U32.p, nn);
  dbgz_count_launch(p->ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_make_Ub(dbgz_problem *p) {
  dbgz_ctx *ctx = p->ctx;
  const int64_t d = p->d, nn = d * d;
  DBGZ_TRY(dbgz_ensure(ctx, p->Ub, sizeof(double) * nn));
  DBGZ_TRY(dbgz_ensure(ctx, p->Ub32, sizeof(float) * nn));
  dim3 g((unsigned)((d + 255) / 256), (unsigned)d);
  k_anti_transpose<<<g, 256, 0, ctx->stream>>>((const double *)p->U.p, d, (double *)p->Ub.p);
  dbgz_count_launch(ctx);
  int blocks = (int)std::min<int64_t>((nn + 255) / 256, 4096);
  k_to_f32<<<blocks, 256, 0, ctx->stream>>>((const double *)p->Ub.p, (float *)p->Ub32.p, nn);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

// chol_dev.cuh -- CTA-level device code of the pivoted blocked Cholesky,
// shared by the one-problem kernels (chol.cu) and the batched factorisation
// (batch.cu): one Genz pivot block and one Schur-update tile.  Arithmetic
// contract as in chol.cu: every sum is one ascending fma chain, every other
// operation one IEEE operation (detmath.h), so all callers give the same
// bits.
#pragma once
#include <cfloat>
#include <cstdint>

#include "detmath.h"

namespace cholk {

// The order findmin/argmin use (Base.isgreater: NaN lowest, -0.0 below +0.0,
// then by value) as an unsigned key: NaN -> 0, otherwise the IEEE bits made
// monotone (negative values complemented, non-negative ones with the sign bit
// set), so -0.0 sorts below +0.0 and equal values give equal keys.  The
// largest key, +inf's, is below ~0, which marks "no candidate".
__device__ __forceinline__ unsigned long long argmin_key(double x) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  if (x != x) return 0ull;
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// The warp's least key and, among the lanes that hold it, the least index
// (ties go to the first candidate, as findmin's do): three warp
// min-reductions on 32-bit words, no compare-and-branch tree.  Lanes without a
// candidate pass key ~0 and index ~0.
__device__ __forceinline__ void warp_argmin(unsigned long long &key, unsigned &idx) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mh = __reduce_min_sync(0xffffffffu, hi);
  const unsigned ml = __reduce_min_sync(0xffffffffu, hi == mh ? lo : 0xffffffffu);
  idx = __reduce_min_sync(0xffffffffu, (hi == mh && lo == ml) ? idx : 0xffffffffu);
  key = ((unsigned long long)mh << 32) | ml;
}

// One bs1 block [i0, i1] of cholesky_genz! inside the bs2 panel ending at
// ii1 (0-based, inclusive), src/cholesky.jl:494-572.  One CTA of up to
// 1024 threads (any multiple of 32).
__device__ __forceinline__ void genz_block_dev(double *M, int64_t n, double *a, double *b, double *dvec,
                                               double *svec, double *ovec, int64_t *perm, int64_t i0,
                                               int64_t i1, int64_t ii1, const double *eps0_ptr, int64_t *rank) {
  __shared__ unsigned long long red_k[32];
  __shared__ unsigned red_t[32];
  __shared__ int64_t sh_im;
  __shared__ double sh_mii, sh_yi;
  __shared__ int sh_stop;
  const double c2 = dm_div(1.0, dm_sqrt(2.0));
  const double is2pi = dm_div(2.0, dm_sqrt(dm_mul(2.0, M_PI)));
  const double eps0 = eps0_ptr[0];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (rank[0] < n) return;  // an earlier block already stopped
  for (int64_t k = i0 + tid; k <= ii1; k += blockDim.x) dvec[k] = 0.0;
  __syncthreads();
  for (int64_t i = i0; i <= i1; ++i) {
    // pivot scores :500-512, then argmin :514
    unsigned long long key = ~0ull;  // this thread's least key, at its first position
    unsigned pos = ~0u;
    for (int64_t k = i + tid; k <= ii1; k += blockDim.x) {
      double m_kk = dm_sub(M[k * n + k], dvec[k]);
      m_kk = m_kk < 0 ? 0.0 : dm_sqrt(m_kk);
      double a_k = dm_mul(dm_div(dm_sub(a[k], svec[k]), m_kk), c2);
      double b_k = dm_mul(dm_div(dm_sub(b[k], svec[k]), m_kk), c2);
      double o = dm_sub(det_erf(b_k), det_erf(a_k));
      ovec[k] = o;
      const unsigned long long ko = argmin_key(o);
      if (ko < key) {
        key = ko;
        pos = (unsigned)(k - i0);
      }
    }
    warp_argmin(key, pos);
    if (lane == 0) {
      red_k[wid] = key;
      red_t[wid] = pos;
    }
    __syncthreads();
    if (wid == 0) {
      const int nw = (int)(blockDim.x >> 5);
      key = lane < nw ? red_k[lane] : ~0ull;
      pos = lane < nw ? red_t[lane] : ~0u;
      warp_argmin(key, pos);
    }
    if (tid == 0) {
      const int64_t im = i0 + (int64_t)pos;
      double d_ii = ovec[im];
      double m_ii = dm_sub(M[im * n + im], dvec[im]);
      if (im != i) {  // :518-523
        int64_t tp = perm[i]; perm[i] = perm[im]; perm[im] = tp;
        double t;
        t = dvec[im]; dvec[im] = dvec[i]; dvec[i] = t;
        t = svec[im]; svec[im] = svec[i]; svec[i] = t;
        t = a[im]; a[im] = a[i]; a[i] = t;
        t = b[im]; b[im] = b[i]; b[i] = t;
      }
      sh_im = im;
      sh_mii = m_ii;
      sh_yi = d_ii;  // carried to the y_i step
    }
    __syncthreads();
    const int64_t im = sh_im;
    if (im != i) {  // :525-530: rows over columns i0..n, then full columns
      for (int64_t k = i0 + tid; k < n; k += blockDim.x) {
        double t = M[k * n + i];
        M[k * n + i] = M[k * n + im];
        M[k * n + im] = t;
      }
      __syncthreads();
      for (int64_t k = tid; k < n; k += blockDim.x) {
        double t = M[i * n + k];
        M[i * n + k] = M[im * n + k];
        M[im * n + k] = t;
      }
      __syncthreads();
    }
    if (tid == 0) {
      double m_ii = sh_mii;
      double d_ii = sh_yi;
      int stop = 0;
      if (m_ii > eps0) {
        m_ii = dm_sqrt(m_ii);
      } else {
        rank[0] = i;  // 0-based i == reference's i - 1
        stop = 1;
      }
      if (!stop) {
        M[i * n + i] = m_ii;
        double a_norm = dm_div(dm_sub(a[i], svec[i]), m_ii);
        double b_norm = dm_div(dm_sub(b[i], svec[i]), m_ii);
        double ea = det_exp(dm_div(-dm_mul(a_norm, a_norm), 2.0));
        double eb = det_exp(dm_div(-dm_mul(b_norm, b_norm), 2.0));
        sh_yi = dm_div(dm_mul(dm_sub(ea, eb), is2pi), d_ii);
        sh_mii = m_ii;
      }
      sh_stop = stop;
    }
    __syncthreads();
    if (sh_stop) return;
    const double m_ii = sh_mii, y_i = sh_yi;
    if (i == i0) {  // :547-554
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        double m_ij = dm_div(M[j * n + i], m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        dvec[j] = dm_add(dvec[j], dm_mul(m_ij, m_ij));
        svec[j] = dm_add(svec[j], dm_mul(y_i, m_ij));
      }
    } else if (i < ii1) {  // :555-570
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        double acc = 0.0;
        for (int64_t l = i0; l <= i - 1; ++l) acc = dm_fma(M[l * n + j], M[i * n + l], acc);
        double m_ij = dm_div(dm_sub(M[i * n + j], acc), m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        dvec[j] = dm_add(dvec[j], dm_mul(m_ij, m_ij));
        svec[j] = dm_add(svec[j], dm_mul(y_i, m_ij));
      }
    }
    __syncthreads();
  }
}

// genz_block_dev with the panel's per-candidate vectors held in shared
// memory for the whole block: dvec, svec, a, b, perm and the diagonal of M
// over [i0, ii1] (sh: 7 (ii1 - i0 + 1) words, see genz_block_smem_bytes).
// The pivot step's serial part (argmin, swaps, the pivot's own terms) then
// makes no global round trips; M's rows and columns stay in global memory.
// Same operations in the same order as genz_block_dev: the same bits.
__host__ __device__ inline size_t genz_block_smem_bytes(int64_t panel_len) { return (size_t)56 * panel_len; }

__device__ __forceinline__ void genz_block_smem(double *M, int64_t n, double *a, double *b, double *dvec,
                                                double *svec, int64_t *perm, int64_t i0, int64_t i1, int64_t ii1,
                                                const double *eps0_ptr, int64_t *rank, double *sh) {
  __shared__ unsigned long long red_k[32];
  __shared__ unsigned red_t[32];
  __shared__ int64_t sh_im;
  __shared__ double sh_mii, sh_yi;
  __shared__ int sh_stop;
  const double c2 = dm_div(1.0, dm_sqrt(2.0));
  const double is2pi = dm_div(2.0, dm_sqrt(dm_mul(2.0, M_PI)));
  const double eps0 = eps0_ptr[0];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (rank[0] < n) return;  // an earlier block already stopped
  const int64_t len = ii1 - i0 + 1;
  double *s_d = sh, *s_s = sh + len, *s_a = sh + 2 * len, *s_b = sh + 3 * len, *s_g = sh + 4 * len,
         *s_o = sh + 5 * len;
  int64_t *s_p = reinterpret_cast<int64_t *>(sh + 6 * len);
  for (int64_t k = tid; k < len; k += blockDim.x) {
    const int64_t g = i0 + k;
    s_d[k] = 0.0;
    s_s[k] = svec[g];
    s_a[k] = a[g];
    s_b[k] = b[g];
    s_g[k] = M[g * n + g];
    s_p[k] = perm[g];
  }
  __syncthreads();
  auto write_back = [&]() {
    __syncthreads();
    for (int64_t k = tid; k < len; k += blockDim.x) {
      const int64_t g = i0 + k;
      dvec[g] = s_d[k];
      svec[g] = s_s[k];
      a[g] = s_a[k];
      b[g] = s_b[k];
      perm[g] = s_p[k];
    }
  };
  for (int64_t i = i0; i <= i1; ++i) {
    // pivot scores :500-512, then argmin :514
    unsigned long long key = ~0ull;  // this thread's least key, at its first position
    unsigned pos = ~0u;
    for (int64_t k = i + tid; k <= ii1; k += blockDim.x) {
      const int64_t q = k - i0;
      double m_kk = dm_sub(s_g[q], s_d[q]);
      m_kk = m_kk < 0 ? 0.0 : dm_sqrt(m_kk);
      double a_k = dm_mul(dm_div(dm_sub(s_a[q], s_s[q]), m_kk), c2);
      double b_k = dm_mul(dm_div(dm_sub(s_b[q], s_s[q]), m_kk), c2);
      double o = dm_sub(det_erf(b_k), det_erf(a_k));
      s_o[q] = o;
      const unsigned long long ko = argmin_key(o);
      if (ko < key) {
        key = ko;
        pos = (unsigned)q;
      }
    }
    warp_argmin(key, pos);
    if (lane == 0) {
      red_k[wid] = key;
      red_t[wid] = pos;
    }
    __syncthreads();
    if (wid == 0) {
      // the warps' minima reduced by warp 0 (the key order with the position
      // as tie-break is a strict total order: the same pivot in any grouping)
      const int nw = (int)(blockDim.x >> 5);
      key = lane < nw ? red_k[lane] : ~0ull;
      pos = lane < nw ? red_t[lane] : ~0u;
      warp_argmin(key, pos);
      const int64_t im = i0 + (int64_t)pos;
      if (lane == 0) {
      const int64_t qi = i - i0, qm = im - i0;
      double d_ii = s_o[qm];
      double m_ii = dm_sub(s_g[qm], s_d[qm]);
      if (im != i) {  // :518-523 (and the diagonal, which the row/column swap moves)
        int64_t tp = s_p[qi]; s_p[qi] = s_p[qm]; s_p[qm] = tp;
        double t;
        t = s_d[qm]; s_d[qm] = s_d[qi]; s_d[qi] = t;
        t = s_s[qm]; s_s[qm] = s_s[qi]; s_s[qi] = t;
        t = s_a[qm]; s_a[qm] = s_a[qi]; s_a[qi] = t;
        t = s_b[qm]; s_b[qm] = s_b[qi]; s_b[qi] = t;
        t = s_g[qm]; s_g[qm] = s_g[qi]; s_g[qi] = t;
      }
      sh_im = im;
      sh_mii = m_ii;
      sh_yi = d_ii;  // carried to the y_i step
      }
    }
    __syncthreads();
    const int64_t im = sh_im;
    // the y_i step (:533-546) by the block's last thread, which has no element
    // of the swap below when n < blockDim: its arithmetic overlaps the swap,
    // its write of the diagonal waits for it (same operations as in order)
    const bool yt = tid == (int)blockDim.x - 1;
    double y_mii = 0.0;
    int y_stop = 0;
    if (yt) {
      double m_ii = sh_mii;
      double d_ii = sh_yi;
      if (m_ii > eps0) {
        m_ii = dm_sqrt(m_ii);
      } else {
        rank[0] = i;  // 0-based i == reference's i - 1
        y_stop = 1;
      }
      if (!y_stop) {
        const int64_t qi = i - i0;
        double a_norm = dm_div(dm_sub(s_a[qi], s_s[qi]), m_ii);
        double b_norm = dm_div(dm_sub(s_b[qi], s_s[qi]), m_ii);
        double ea = det_exp(dm_div(-dm_mul(a_norm, a_norm), 2.0));
        double eb = det_exp(dm_div(-dm_mul(b_norm, b_norm), 2.0));
        sh_yi = dm_div(dm_mul(dm_sub(ea, eb), is2pi), d_ii);
        sh_mii = m_ii;
      }
      sh_stop = y_stop;
      y_mii = m_ii;
    }
    if (im != i) {
      // :525-530, rows i <-> im over columns i0..n-1, then columns i <-> im,
      // in one pass: for k outside {i, im} the two swaps touch four distinct
      // elements; the 2 x 2 block on {i, im} ends up as (i,i) <- (im,im),
      // (im,im) <- (i,i), (i,im) <- (im,i), (im,i) <- (i,im)
      for (int64_t k = tid; k < n; k += blockDim.x) {
        if (k == i || k == im) {
          if (k == i) {
            const double ii = M[i * n + i], mm = M[im * n + im], im_i = M[i * n + im], i_im = M[im * n + i];
            M[i * n + i] = mm;
            M[im * n + im] = ii;
            M[im * n + i] = im_i;
            M[i * n + im] = i_im;
          }
          continue;
        }
        if (k >= i0) {
          const double t = M[k * n + i];
          M[k * n + i] = M[k * n + im];
          M[k * n + im] = t;
        }
        const double t = M[i * n + k];
        M[i * n + k] = M[im * n + k];
        M[im * n + k] = t;
      }
      __syncthreads();
    }
    if (yt && !y_stop) M[i * n + i] = y_mii;
    __syncthreads();
    if (sh_stop) {
      write_back();
      return;
    }
    const double m_ii = sh_mii, y_i = sh_yi;
    if (i == i0) {  // :547-554
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        const int64_t q = j - i0;
        double m_ij = dm_div(M[j * n + i], m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        s_d[q] = dm_add(s_d[q], dm_mul(m_ij, m_ij));
        s_s[q] = dm_add(s_s[q], dm_mul(y_i, m_ij));
      }
    } else if (i < ii1) {  // :555-570
      for (int64_t j = i + 1 + tid; j <= ii1; j += blockDim.x) {
        const int64_t q = j - i0;
        // the ascending fma chain over l, its operands loaded 8 at a time
        // ahead of the chain
        double acc = 0.0;
        int64_t l = i0;
        for (; l + 8 <= i; l += 8) {
          double x[8], y[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            x[u] = M[(l + u) * n + j];
            y[u] = M[i * n + l + u];
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) acc = dm_fma(x[u], y[u], acc);
        }
        for (; l <= i - 1; ++l) acc = dm_fma(M[l * n + j], M[i * n + l], acc);
        double m_ij = dm_div(dm_sub(M[i * n + j], acc), m_ii);
        M[j * n + i] = m_ij;
        M[i * n + j] = m_ij;
        s_d[q] = dm_add(s_d[q], dm_mul(m_ij, m_ij));
        s_s[q] = dm_add(s_s[q], dm_mul(y_i, m_ij));
      }
    }
    __syncthreads();
  }
  write_back();
}

// genz_block_smem with the block's factor entries kept on chip.  The entries
// m[l, k] of the block's pivots l for every candidate k of the panel, which
// the row update's dot products read, live in the registers of the
// candidate's thread (the first kFReg pivots) and in shared memory (the rest),
// and follow their candidate through the swaps.  Thread t < kOnchipSlots owns
// panel position i0 + t; it takes the value M[i, k] its update needs while it
// does its part of the row/column swap, so the pivot chain makes no global
// read but that one.  A last warp computes y_i (:533-546) while the slot
// threads run the update's dot products (named barrier 2: y_i ready).  Panels
// of at most kOnchipSlots positions, blocks of at most kOnchipPiv pivots.  Same
// operations in the same order as genz_block_dev: the same bits.
constexpr int kFReg = 16;          // block pivots whose entries live in registers
constexpr int kOnchipPiv = 64;     // pivots per block at most
constexpr int kOnchipSlots = 512;  // slot threads; the block has one more warp
constexpr int kSwapBatch = 2;      // swap indices per memory round trip
__host__ __device__ inline size_t genz_block_onchip_bytes(int64_t panel_len) {
  return (size_t)(56 + 8 * (kOnchipPiv - kFReg)) * (size_t)panel_len + 8 * 2 * kFReg;
}
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ void named_bar_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void genz_block_onchip(double *M, int64_t n, double *a, double *b, double *dvec,
                                                  double *svec, int64_t *perm, int64_t i0, int64_t i1,
                                                  int64_t ii1, const double *eps0_ptr, int64_t *rank, double *sh) {
  __shared__ unsigned long long red_k[32];
  __shared__ unsigned red_t[32];
  __shared__ double sh_yi, sh_mij_im;
  const double c2 = dm_div(1.0, dm_sqrt(2.0));
  const double is2pi = dm_div(2.0, dm_sqrt(dm_mul(2.0, M_PI)));
  const double eps0 = eps0_ptr[0];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NS = kOnchipSlots, NALL = kOnchipSlots + 32;
  if (rank[0] < n) return;  // an earlier block already stopped
  const int64_t len = ii1 - i0 + 1;
  double *s_d = sh, *s_s = sh + len, *s_a = sh + 2 * len, *s_b = sh + 3 * len, *s_g = sh + 4 * len,
         *s_o = sh + 5 * len;
  int64_t *s_p = reinterpret_cast<int64_t *>(sh + 6 * len);
  double *s_f = sh + 7 * len;                        // [kOnchipPiv - kFReg][len]: pivots kFReg.. of each position
  double *s_piv = s_f + (kOnchipPiv - kFReg) * len;  // the pivot's register entries
  double *s_x = s_piv + kFReg;                       // the displaced candidate's register entries
  for (int64_t k = tid; k < len; k += blockDim.x) {
    const int64_t g = i0 + k;
    s_d[k] = 0.0;
    s_s[k] = svec[g];
    s_a[k] = a[g];
    s_b[k] = b[g];
    s_g[k] = M[g * n + g];
    s_p[k] = perm[g];
  }
  __syncthreads();
  auto write_back = [&]() {
    __syncthreads();
    for (int64_t k = tid; k < len; k += blockDim.x) {
      const int64_t g = i0 + k;
      dvec[g] = s_d[k];
      svec[g] = s_s[k];
      a[g] = s_a[k];
      b[g] = s_b[k];
      perm[g] = s_p[k];
    }
  };
  const bool yw = wid == NS / 32;  // the y_i warp
  const int t = tid;               // this thread's panel position: kk = i0 + t
  const bool has_slot = !yw && t < len;
  const int64_t kk = i0 + t;
  double f[kFReg];                 // m[i0 + u, kk] for u < kFReg
#pragma unroll
  for (int u = 0; u < kFReg; ++u) f[u] = 0.0;
  double mij = 0.0;                // M[i, kk] of the coming update
  // pivot score of this position for step i (:500-512), and the warp's minimum
  auto score = [&](int64_t i) {
    unsigned long long key = ~0ull;
    unsigned pos = ~0u;
    if (has_slot && kk >= i) {
      double m_kk = dm_sub(s_g[t], s_d[t]);
      m_kk = m_kk < 0 ? 0.0 : dm_sqrt(m_kk);
      double a_k = dm_mul(dm_div(dm_sub(s_a[t], s_s[t]), m_kk), c2);
      double b_k = dm_mul(dm_div(dm_sub(s_b[t], s_s[t]), m_kk), c2);
      double o = dm_sub(det_erf(b_k), det_erf(a_k));
      s_o[t] = o;
      key = argmin_key(o);
      pos = (unsigned)t;
    }
    warp_argmin(key, pos);
    if (lane == 0) {
      red_k[wid] = key;
      red_t[wid] = pos;
    }
  };
  for (int64_t i = i0; i <= i1; ++i) {
    const int np = (int)(i - i0);  // block pivots before i
    // one call site of the scores (their special functions are long code)
    if (!yw) score(i);
    __syncthreads();
    // every warp reduces the warps' minima itself (the key order with the
    // position as tie-break is a strict total order: the same pivot in each)
    unsigned long long key = lane < NS / 32 ? red_k[lane] : ~0ull;
    unsigned pos = lane < NS / 32 ? red_t[lane] : ~0u;
    warp_argmin(key, pos);
    const int qm = (int)pos;
    const int64_t im = i0 + qm;
    const double m_raw = dm_sub(s_g[qm], s_d[qm]);
    const bool stop = !(m_raw > eps0);  // the rank test of :533-537
    const double m_pp = stop ? 0.0 : dm_sqrt(m_raw);
    if (yw) {
      // y_i (:538-546) while the slot threads swap and update
      // (the pivot's values are read at qm, before its swap with position np)
      if (lane == 0) {
        if (stop) {
          rank[0] = i;  // 0-based i == reference's i - 1
        } else {
          double a_norm = dm_div(dm_sub(s_a[qm], s_s[qm]), m_pp);
          double b_norm = dm_div(dm_sub(s_b[qm], s_s[qm]), m_pp);
          double ea = det_exp(dm_div(-dm_mul(a_norm, a_norm), 2.0));
          double eb = det_exp(dm_div(-dm_mul(b_norm, b_norm), 2.0));
          sh_yi = dm_div(dm_mul(dm_sub(ea, eb), is2pi), s_o[qm]);
        }
      }
      __syncwarp();
      named_bar_arrive(1, NALL);  // its reads of position qm are done
      if (stop) {
        write_back();
        return;
      }
      named_bar_arrive(2, NALL);
    } else {
      // :518-523, the per-position values of np and qm trade places after
      // barrier 1, when every read of them for this step is done: d and s,
      // which the displaced candidate's update uses next, by the two threads
      // (each takes the other's now and stores its own), the rest by thread np
      const bool swp = im != i && (t == np || t == qm);
      double x_d = 0.0, x_s = 0.0;
      if (swp) {
        const int o2 = t == np ? qm : np;
        x_d = s_d[o2];
        x_s = s_s[o2];
      }
      // the pivot's register entries for every candidate's dot product, the
      // displaced candidate's for its new position
      if (t == qm) {
#pragma unroll
        for (int u = 0; u < kFReg; ++u) s_piv[u] = f[u];
      }
      if (im != i && t == np) {
#pragma unroll
        for (int u = 0; u < kFReg; ++u) s_x[u] = f[u];
      }
      if (im != i) {
        // the shared-memory entries of the two positions trade places
        for (int u = kFReg + t; u < np; u += NS) {
          double *row = s_f + (int64_t)(u - kFReg) * len;
          const double tt = row[np];
          row[np] = row[qm];
          row[qm] = tt;
        }
        // :525-530, rows i <-> im over columns i0..n-1, then columns i <-> im,
        // in one pass: for k outside {i, im} the two swaps touch four distinct
        // elements; the 2 x 2 block on {i, im} ends up as (i,i) <- (im,im),
        // (im,im) <- (i,i), (i,im) <- (im,i), (im,i) <- (i,im), and (i,i)
        // then takes the pivot m_ii.  Position k's thread does index k
        // (k >= i0), so it keeps the value its update reads: M[k, i] after the
        // swap, or M[i, k] for the block's first pivot.  This thread's indices
        // are its own position i0 + t, then the indices outside the panel
        // ([0, i0) and (ii1, n), numbered o = 0, 1, ...) o = t + e NS:
        // kSwapBatch of them at a time, all loaded before any is stored (no
        // element is shared between threads), so the swap costs one memory
        // round trip per batch -- one in all when n <= len + NS.
        const int64_t nOwn = has_slot ? 1 : 0;
        const int64_t nOut = t < n - len ? (n - len - t + NS - 1) / NS : 0;
        for (int64_t e0 = 0; e0 < nOwn + nOut; e0 += kSwapBatch) {
          auto kidx = [&](int e) -> int64_t {
            const int64_t q = e0 + e;
            if (q < nOwn) return kk;
            if (q >= nOwn + nOut) return -1;
            const int64_t o = t + (q - nOwn) * NS;
            return o < i0 ? o : o + len;
          };
          double ri[kSwapBatch], rm[kSwapBatch], ci[kSwapBatch], cm[kSwapBatch];
          bool diag = false;
#pragma unroll
          for (int e = 0; e < kSwapBatch; ++e) {
            const int64_t k = kidx(e);
            diag = diag || k == i;
            const bool live = k >= 0 && k != i && k != im, row = live && k >= i0;
            ri[e] = row ? M[k * n + i] : 0.0;
            rm[e] = row ? M[k * n + im] : 0.0;
            ci[e] = live ? M[i * n + k] : 0.0;
            cm[e] = live ? M[im * n + k] : 0.0;
          }
          double d_ii = 0.0, d_mm = 0.0, d_mi = 0.0, d_im = 0.0;
          if (diag) {
            d_ii = M[i * n + i];
            d_mm = M[im * n + im];
            d_mi = M[i * n + im];
            d_im = M[im * n + i];
          }
#pragma unroll
          for (int e = 0; e < kSwapBatch; ++e) {
            const int64_t k = kidx(e);
            const bool live = k >= 0 && k != i && k != im, row = live && k >= i0;
            if (row) {
              M[k * n + i] = rm[e];
              M[k * n + im] = ri[e];
            }
            if (live) {
              M[i * n + k] = cm[e];
              M[im * n + k] = ci[e];
              if (k == kk) mij = np == 0 ? rm[e] : cm[e];
            }
          }
          if (diag) {
            M[i * n + i] = stop ? d_mm : m_pp;
            M[im * n + im] = d_ii;
            M[im * n + i] = d_mi;
            M[i * n + im] = d_im;
            sh_mij_im = np == 0 ? d_mi : d_im;  // for position im
          }
        }
      } else {
        if (has_slot && kk > i) mij = np == 0 ? M[kk * n + i] : M[i * n + kk];
        if (t == np && !stop) M[i * n + i] = m_pp;
      }
      named_bar_sync(1, NALL);
      if (swp) {
        s_d[t] = x_d;
        s_s[t] = x_s;
        if (t == np) {
          const int64_t tp = s_p[np]; s_p[np] = s_p[qm]; s_p[qm] = tp;
          double tt;
          tt = s_a[np]; s_a[np] = s_a[qm]; s_a[qm] = tt;
          tt = s_b[np]; s_b[np] = s_b[qm]; s_b[qm] = tt;
          tt = s_g[np]; s_g[np] = s_g[qm]; s_g[qm] = tt;
        }
      }
      if (im != i) {
        if (t == np) {
#pragma unroll
          for (int u = 0; u < kFReg; ++u) f[u] = s_piv[u];
        } else if (t == qm) {
#pragma unroll
          for (int u = 0; u < kFReg; ++u) f[u] = s_x[u];
          mij = sh_mij_im;
        }
      }
      if (stop) {
        write_back();
        return;
      }
      // the update of step i (:547-570) for this position
      const bool upd = has_slot && kk > i;
      double m = 0.0;
      if (upd) {
        if (np == 0) {
          m = dm_div(mij, m_pp);
        } else {
          // the ascending fma chain over the block's pivots l = i0 .. i - 1
          double acc = 0.0;
#pragma unroll
          for (int u = 0; u < kFReg; ++u)
            if (u < np) acc = dm_fma(f[u], s_piv[u], acc);
          int u = kFReg;
          for (; u + 8 <= np; u += 8) {
            double x[8], y[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const double *row = s_f + (int64_t)(u + e - kFReg) * len;
              x[e] = row[t];
              y[e] = row[np];
            }
#pragma unroll
            for (int e = 0; e < 8; ++e) acc = dm_fma(x[e], y[e], acc);
          }
          for (; u < np; ++u) {
            const double *row = s_f + (int64_t)(u - kFReg) * len;
            acc = dm_fma(row[t], row[np], acc);
          }
          m = dm_div(dm_sub(mij, acc), m_pp);
        }
        s_d[t] = dm_add(s_d[t], dm_mul(m, m));
        if (np < kFReg) {
#pragma unroll
          for (int u2 = 0; u2 < kFReg; ++u2) f[u2] = u2 == np ? m : f[u2];
        } else {
          s_f[(int64_t)(np - kFReg) * len + t] = m;
        }
        M[kk * n + i] = m;
        M[i * n + kk] = m;
      }
      named_bar_sync(2, NALL);  // y_i
      if (upd) s_s[t] = dm_add(s_s[t], dm_mul(sh_yi, m));
    }
  }
  write_back();
}

// C[j,k] -= sum_{l=p0..p1} A(l,j) * B(l,k) for j,k in [c0, c1], one
// ascending fma chain per element.  A(l,j) = M[j,l] (row form, the
// reference's lower-triangle copy) when a_row, else M[l,j]; B(l,k) = M[l,k].
// One 32 x 32 output tile (j0, k0) per call, 256 threads (32 x 8).
constexpr int kTile = 32;
__device__ __forceinline__ void schur_tile_dev(double *M, int64_t n, int64_t p0, int64_t p1, int64_t c0,
                                               int64_t c1, int a_row, int64_t j0, int64_t k0) {
  __shared__ double As[kTile][kTile + 1];
  __shared__ double Bs[kTile][kTile + 1];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t l0 = p0; l0 <= p1; l0 += kTile) {
    for (int r = ty; r < kTile; r += 8) {
      // As[l][c] = A(l0 + l, j0 + c); Bs[l][c] = B(l0 + l, k0 + c)
      int64_t l = l0 + tx, jj = j0 + r, kk = k0 + r;
      if (a_row) {
        int64_t lr = l0 + r, jc = j0 + tx;  // coalesced over j
        As[r][tx] = (lr <= p1 && jc <= c1) ? M[lr * n + jc] : 0.0;
      } else {
        As[tx][r] = (l <= p1 && jj <= c1) ? M[jj * n + l] : 0.0;
      }
      Bs[tx][r] = (l <= p1 && kk <= c1) ? M[kk * n + l] : 0.0;
    }
    __syncthreads();
    const int lmax = (int)((p1 - l0 + 1) < kTile ? (p1 - l0 + 1) : kTile);
    for (int l = 0; l < lmax; ++l) {
      double av = As[l][tx];
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[r] = dm_fma(av, Bs[l][ty + 8 * r], acc[r]);
    }
    __syncthreads();
  }
  const int64_t j = j0 + tx;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    int64_t k = k0 + ty + 8 * r;
    if (j <= c1 && k <= c1) M[k * n + j] = dm_sub(M[k * n + j], acc[r]);
  }
}

}  // namespace cholk

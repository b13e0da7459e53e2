// du_gemm.cu -- the factor gradient of the FP32 gradient modes on tcgen05:
//
//   dU[l, t] (+)= sum_n Y[l][n] S[t][n]     for l < t only,
//
// where Y (the stored y's) and S (the stored p * sbar) are FP32 arrays in
// the tile-major layout of the gradient state: [tile][row < d][128 samples],
// nc samples.
// Only the strict upper triangle of dU enters the gradient, so only the
// output tiles that hold some l < t are computed (20 of 32 at d = 1000).
//
// Tiles of 128 (l) x 256 (t); the 32-sample chunks are dealt to the CTAs of
// a tile round robin (split-K: split s takes chunks s, s + S, s + 2S, ...)
// so that the few tiles fill the GPU, and the splits of one tile are summed
// afterwards in a fixed order (deterministic).  Per CTA: warp 5 streams
// 32-sample K-major stages of Y rows and S rows by TMA (128-byte swizzle,
// 4 stages), warp 4 issues kind::tf32 MMAs (M = 128, N = 256, K = 8) into a
// TMEM accumulator, warps 0-3 read the accumulator back and write the
// CTA's partial tile.  With the chunks interleaved, every CTA streams through
// the same sample window at about the same time, so the rows that several
// tiles share come from L2: the arrays are read from HBM about once (16.8 GB
// at d = 1000, 2^21 samples) instead of once per tile (contiguous sample
// ranges per split drifted apart at that size and read them 3-4 times).
// Every wait is bounded (sm100.cuh).
//
// The inputs are FP32 in memory and the tensor cores read them as TF32
// (the low 13 mantissa bits are not used), as a TF32 library GEMM does.
#include <cuda.h>
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "sm100.cuh"

namespace {

using namespace sm100;

constexpr int TM = 128, TN = 256, KC = 32, STAGES = 4;
constexpr int NT = 192;  // 4 epilogue warps, MMA warp, TMA warp
constexpr int kMmaWarp = 4, kProdWarp = 5;
constexpr int ABYTES = TM * KC * 4, BBYTES = TN * KC * 4;  // 16 KB, 32 KB per stage
constexpr int SMEM = STAGES * (ABYTES + BBYTES) + 1024 + 1024;

struct __align__(64) DuParams {
  CUtensorMap tm_y, tm_s;
  int64_t nk;       // 32-sample chunks in total
  int n_tiles, n_split;
  const int32_t *tile_l0, *tile_t0;
  float *work;      // [split][tile][128][256]
  int *status;
};

struct DuMisc {
  uint64_t full[STAGES], empty[STAGES], done;
  uint32_t tmem_base;
  int abort;
};

__global__ void __launch_bounds__(NT, 1) k_du_gemm(const __grid_constant__ DuParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *abuf = sm, *bbuf = sm + STAGES * ABYTES;
  DuMisc *ms = reinterpret_cast<DuMisc *>(sm + STAGES * (ABYTES + BBYTES));
  volatile int *abort = &ms->abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x, split = blockIdx.y;
  const int32_t l0 = P.tile_l0[tile], t0 = P.tile_t0[tile];
  // the chunks of this split: split, split + n_split, ... (interleaved, so that
  // all CTAs stream through the same sample window at the same time and the
  // rows they share are found in L2)
  const int64_t nkc = (P.nk - split + P.n_split - 1) / P.n_split;

  if (tid == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&ms->full[i], 1);
      mbar_init(&ms->empty[i], 1);
    }
    mbar_init(&ms->done, 1);
    ms->abort = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(&ms->tmem_base, (uint32_t)TN);
    tmem_relinquish();
  }
  if (warp == kProdWarp && lane == 0) {
    prefetch_tmap(&P.tm_y);
    prefetch_tmap(&P.tm_s);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = ms->tmem_base;

  if (warp == kProdWarp) {
    if (lane == 0) {
      bool ok = true;
      int64_t i = 0;
      for (; i < nkc && ok; ++i) {
        const int s = (int)(i % STAGES);
        if (i >= STAGES) ok = mbar_wait(&ms->empty[s], (uint32_t)((i / STAGES - 1) & 1), abort);
        if (!ok) break;
        // chunk c = samples 32c..32c+31: tile c / 4, samples 32 (c % 4).. of it
        const int64_t c = split + i * P.n_split;
        const int32_t x = (int32_t)((c & 3) * KC), z = (int32_t)(c >> 2);
        mbar_arrive_expect_tx(&ms->full[s], (uint32_t)(ABYTES + BBYTES));
        tma_load_3d(abuf + s * ABYTES, &P.tm_y, x, l0, z, &ms->full[s]);
        tma_load_3d(bbuf + s * BBYTES, &P.tm_s, x, t0, z, &ms->full[s]);
      }
      if (!ok) {
        ms->abort = 1;
        atomicExch(P.status, DBGZ_ERR_TIMEOUT);
        // let the loads already issued land before the CTA leaves
        for (int64_t j = std::max<int64_t>(0, i - STAGES); j < i; ++j)
          mbar_wait(&ms->full[j % STAGES], (uint32_t)((j / STAGES) & 1), abort);
      }
    }
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      bool ok = true;
      const uint32_t idesc = instr_desc(2, 2, TM, TN);
      for (int64_t i = 0; i < nkc && ok; ++i) {
        const int s = (int)(i % STAGES);
        ok = mbar_wait(&ms->full[s], (uint32_t)((i / STAGES) & 1), abort);
        if (!ok) break;
        tc_fence_after();
        const uint32_t a = smem_u32(abuf + s * ABYTES), b = smem_u32(bbuf + s * BBYTES);
#pragma unroll
        for (int ks = 0; ks < KC / 8; ++ks)
          mma_tf32(tmem, smem_desc(a + 32 * ks, 1024, 2), smem_desc(b + 32 * ks, 1024, 2), idesc,
                   (i > 0 || ks > 0) ? 1u : 0u);
        mma_commit(&ms->empty[s]);
      }
      if (!ok) {
        ms->abort = 1;
        atomicExch(P.status, DBGZ_ERR_TIMEOUT);
      }
      mma_commit(&ms->done);
    }
  } else {
    // epilogue: warp w owns TMEM lanes 32w..32w+31 (rows l0 + 32w + lane)
    bool ok = mbar_wait(&ms->done, 0, abort);
    if (!ok && !*abort) {
      ms->abort = 1;
      atomicExch(P.status, DBGZ_ERR_TIMEOUT);
    }
    if (ok) {
      tc_fence_after();
      const int row = 32 * warp + lane;
      float4 *dst = reinterpret_cast<float4 *>(P.work + (((int64_t)split * P.n_tiles + tile) * TM + row) * TN);
#pragma unroll 1
      for (int c = 0; c < TN / 32; ++c) {
        uint32_t v[32];
        if (nkc > 0) {
          tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * c), v);
          tmem_wait_ld();
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = 0u;  // an empty split contributes zeros
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
          dst[8 * c + j] = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                       __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
      }
    }
  }
  // the MMA warp's last commit covers every MMA: wait for it before freeing TMEM
  if (warp == kMmaWarp && lane == 0) {
    if (!mbar_wait(&ms->done, 0, abort)) {
      const uint64_t tw = globaltimer();
      while (!mbar_try_wait(&ms->done, 0) && globaltimer() - tw < kWaitLimitNs) {
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, (uint32_t)TN);
  }
}

// dU[t*d + l] = (accumulate ? dU : 0) + sum over splits (in split order) of
// the partial tiles, for l < t; other entries are left alone.
__global__ void k_du_reduce(const float *work, int n_split, int n_tiles, const int32_t *tile_of, int ntj,
                            int64_t d, float *dU, int accumulate) {
  const int64_t l = blockIdx.y;  // threads along t: the partial tiles are read contiguously
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (l >= t || t >= d) return;
  const int li = (int)(l / TM), tj = (int)(t / TN);
  const int tile = tile_of[li * ntj + tj];
  const int64_t off = ((int64_t)tile * TM + (l - (int64_t)li * TM)) * TN + (t - (int64_t)tj * TN);
  double acc = 0.0;
  for (int s = 0; s < n_split; ++s) acc += (double)work[(int64_t)s * n_tiles * TM * TN + off];
  const int64_t ix = t * d + l;
  dU[ix] = accumulate ? (float)((double)dU[ix] + acc) : (float)acc;
}

typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                            CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// [tile][row][128 samples] FP32: x = sample in the tile, y = row, z = tile
int encode_rows(dbgz_ctx *ctx, CUtensorMap *m, const float *base, int64_t nc, int64_t rows, uint32_t box_rows) {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeFn)p;
  }
  if (!fn) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[3] = {128, (cuuint64_t)rows, (cuuint64_t)(nc / 128)};
  cuuint64_t strides[2] = {128 * 4, (cuuint64_t)rows * 128 * 4};
  cuuint32_t box[3] = {(cuuint32_t)KC, box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DBGZ_OK;
}

}  // namespace

int dbgz_du_gemm_tf32(dbgz_ctx *ctx, int64_t d, const float *Y, const float *S, int64_t nc, float *dU,
                      bool accumulate, DevBuf &work) {
  if (nc % 128 != 0 || ((uintptr_t)Y & 15) || ((uintptr_t)S & 15))
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "du_gemm: samples must come in whole 128-sample tiles");
  // the output tiles that hold some l < t
  const int nli = (int)((d + TM - 1) / TM), ntj = (int)((d + TN - 1) / TN);
  std::vector<int32_t> l0s, t0s, tile_of((size_t)nli * ntj, -1);
  for (int tj = 0; tj < ntj; ++tj)
    for (int li = 0; li < nli; ++li)
      if ((int64_t)li * TM < (int64_t)tj * TN + TN - 1 && (int64_t)li * TM < d - 1) {
        tile_of[(size_t)li * ntj + tj] = (int32_t)l0s.size();
        l0s.push_back(li * TM);
        t0s.push_back(tj * TN);
      }
  const int n_tiles = (int)l0s.size();
  const int64_t nk = nc / KC;
  const int n_split = (int)std::max<int64_t>(1, std::min<int64_t>(nk, ctx->num_sms / std::max(n_tiles, 1)));
  const size_t wbytes = (size_t)n_split * n_tiles * TM * TN * 4;
  const size_t tbytes = 4 * (3 * (size_t)n_tiles + tile_of.size()) + 256;
  DBGZ_TRY(dbgz_ensure(ctx, work, wbytes + tbytes + 512));
  float *w = (float *)work.p;
  int32_t *tab = (int32_t *)((char *)work.p + ((wbytes + 255) & ~size_t(255)));
  std::vector<int32_t> h(2 * n_tiles + tile_of.size());
  std::copy(l0s.begin(), l0s.end(), h.begin());
  std::copy(t0s.begin(), t0s.end(), h.begin() + n_tiles);
  std::copy(tile_of.begin(), tile_of.end(), h.begin() + 2 * n_tiles);
  cudaStream_t st = ctx->stream;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(tab, h.data(), 4 * h.size(), cudaMemcpyHostToDevice, st));
  DuParams P;
  std::memset(&P, 0, sizeof(P));
  DBGZ_TRY(encode_rows(ctx, &P.tm_y, Y, nc, d, TM));
  DBGZ_TRY(encode_rows(ctx, &P.tm_s, S, nc, d, TN));
  P.nk = nk;
  P.n_tiles = n_tiles;
  P.n_split = n_split;
  P.tile_l0 = tab;
  P.tile_t0 = tab + n_tiles;
  P.work = w;
  P.status = ctx->d_status;
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(k_du_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
  k_du_gemm<<<dim3((unsigned)n_tiles, (unsigned)n_split), NT, SMEM, st>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  k_du_reduce<<<dim3((unsigned)((d + 127) / 128), (unsigned)(d - 1)), 128, 0, st>>>(w, n_split, n_tiles,
                                                                            tab + 2 * n_tiles, ntj, d, dU,
                                                                            accumulate ? 1 : 0);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

// loop_sparse.cu -- the banded / sparse Genz integration loop.
//
// Replaces qmc_loop!(::QMCDataSparse) (reference src/qmc.jl:618-718) and the
// construction of its CSC factor (src/qmc.jl:262-279):
//   U_S = sparse(triu(U, 1)) after the classic (unpivoted) Cholesky and the
//   eps/(9d) truncation; per dimension i the conditioning sum is the CSC dot
//   s = sum_{p in column i+1} y[rowval[p]] * nzval[p] in ascending row order,
//   then the erf-form CDF and weight of the dense loop.
//
// Work decomposition: one thread per sample, 128 samples per CTA, several
// CTAs per SM (no tensor cores: the dot has at most `bandwidth` terms).  The
// y history a sample needs is the last W = bandwidth + 1 values; it lives in
// a shared-memory ring buffer [W][128] when W fits (W <= 257 in FP32, 129 in
// FP64) and otherwise in a per-CTA slot of global memory.  W is not rounded
// to a power of two (at bandwidth 64 that halves the ring and doubles the
// CTAs per SM): the CSC entries of 32 columns are staged in shared memory per
// block of 32 dimensions with their ring slot (row mod W) in place of the row.
// In FP32 the dot runs as 4 interleaved partial sums (the FP64 loop keeps
// the reference's single ascending chain, so that it matches bit for bit).
#include "internal.cuh"
#include "genz_step.cuh"
#include "policies.cuh"
#include <algorithm>
#include <vector>

namespace {

constexpr int TS = 128;
constexpr int CB = 32;  // columns (dimensions) per staged block

template <typename T>
struct TgtT;
template <>
struct TgtT<double> {
  using type = TargetParams64;
};
template <>
struct TgtT<float> {
  using type = TargetParams32;
};

// A staged CSC entry: the offset of its row's ring slot (slot * 128) and its
// value, read together by one shared-memory load.
template <typename T>
struct __align__(sizeof(T) == 4 ? 8 : 16) SlotVal {
  int off;
  T val;
};

template <typename T>
struct SparseParams {
  int64_t d, nY, m, n_reps, tiles_per_shift, n_tiles;
  dbgz::GenParams gen;
  const int64_t *colptr;   // d + 1
  const int32_t *rowval;   // nnz
  const T *nzval;          // nnz
  const typename TgtT<T>::type *tgt;
  double c1, dc1, up1;
  double *partials;
  T *yglob;                // global ring slots (gridDim.x x W x TS) when W is large
  int W;                   // ring size (bandwidth + 1)
  int ring_in_smem;
  int max_block_nnz;       // staging capacity (entries)
  int64_t tile0;           // tiles [tile0, n_tiles) of the pass
  pol::GradIO<T> io;
  // dimension segments (PassArgs, internal.cuh): y-indices [i_begin, i_end),
  // checkpoint restore / save of the ring and the recursion state
  int64_t i_begin, i_end;
  int ck_load, ck_save, tile_finish;
  const T *ck_in_ring;
  const double *ck_in_state;
  T *ck_ring;
  double *ck_state;
  int64_t ck_seg, ck_N;
};

// Policy: pol::Forward<T, GEN, STORE> or pol::Adjoint<T, GEN> (policies.cuh);
// the adjoint runs on the CSC of the anti-transposed factor.
template <typename T, typename Policy>
__global__ void __launch_bounds__(TS) k_genz_sparse(const SparseParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // layout: [staged entries x cap][colptr of block (CB+1)][ring].  The staged
  // entries are (slot offset, value) pairs, read by one load each, or -- in
  // the FP32 forward pass without stored state -- two arrays of offsets and
  // values (measured on the banded d = 10^4, bandwidth 64, 2^18 x 10 Sobol
  // workload: pairs 947 ms, arrays 863 ms for that pass; pairs
  // faster for the FP64 pass, 1552 against 1588 ms, and the FP32 gradient,
  // 1744 against 2002 ms)
  constexpr bool kPairs = sizeof(T) == 8 || !Policy::kPlain;
  SlotVal<T> *sent = reinterpret_cast<SlotVal<T> *>(smem_raw);
  int32_t *soff = reinterpret_cast<int32_t *>(smem_raw);
  T *sval = reinterpret_cast<T *>(smem_raw + ((sizeof(int32_t) * P.max_block_nnz + 15) & ~size_t(15)));
  int *scol = reinterpret_cast<int *>(smem_raw + ((sizeof(SlotVal<T>) * P.max_block_nnz + 15) & ~size_t(15)));
  T *ring = reinterpret_cast<T *>(scol + CB + 4);
  __shared__ pol::Staged<T> sg;
  __shared__ uint32_t sob[Policy::kSobolTable ? CB : 1][dbgz::kSobolRow];  // Sobol integers of the block (dbgz::sobol_stage_block)
  __shared__ double red[TS / 32];
  const int r = threadIdx.x;
  const int W = P.W;
  T *yr = P.ring_in_smem ? ring : P.yglob + (int64_t)blockIdx.x * P.W * TS;

  for (int64_t tile = P.tile0 + blockIdx.x; tile < P.n_tiles; tile += gridDim.x) {
    const int64_t k = tile / P.tiles_per_shift;
    const int64_t j = (tile - k * P.tiles_per_shift) * TS + r;
    Policy pl;
    pl.tile_begin(P.gen, P.d, tile, P.tiles_per_shift, r, P.c1, P.dc1, P.up1, 0, P.io);
    // this row's terms of the staged Sobol integers of the tile
    const dbgz::SobolLane sob_lane(r, (uint64_t)(P.gen.sobol_first + pl.gen.gen_base + (j - r)));
    const int64_t gck = (tile - P.tile0) * TS + r;  // this sample's checkpoint column
    // save / restore of the ring (slot order) and the recursion state
    auto ck_store = [&](T *ring_out, double *state_out) {
      for (int w = 0; w < W; ++w) ring_out[(int64_t)w * P.ck_N + gck] = yr[w * TS + r];
      double v[4];
      pl.pack(v);
#pragma unroll
      for (int e = 0; e < 4; ++e) state_out[(int64_t)e * P.ck_N + gck] = v[e];
    };
    int wslot = 0;  // ring slot of y-index i (i mod W)
    if (P.ck_load) {
      for (int w = 0; w < W; ++w) yr[w * TS + r] = P.ck_in_ring[(int64_t)w * P.ck_N + gck];
      double v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = P.ck_in_state[(int64_t)e * P.ck_N + gck];
      pl.unpack(v);
      wslot = (int)(P.i_begin % W);
    }
    for (int64_t i0 = P.i_begin; i0 < P.i_end; i0 += CB) {
      const int nb = (int)(P.i_end - i0 < CB ? P.i_end - i0 : CB);
      // stage the CSC columns i0+1 .. i0+nb (targets of y-indices i0..i0+nb-1)
      __syncthreads();
      const int64_t p0 = P.colptr[i0 + 1], p1 = P.colptr[i0 + nb + 1];
      const int cnt = (int)(p1 - p0);
      const bool staged = cnt <= P.max_block_nnz;
      if (staged)
        for (int e = r; e < cnt; e += TS) {
          const int off = (P.rowval[p0 + e] % W) * TS;  // the row's ring slot
          if (kPairs) {
            sent[e].off = off;
            sent[e].val = P.nzval[p0 + e];
          } else {
            soff[e] = off;
            sval[e] = P.nzval[p0 + e];
          }
        }
      if (r <= nb) scol[r] = (int)(P.colptr[i0 + 1 + r] - p0);
      pl.stage(sg, P.tgt, r, i0, nb);
      if constexpr (Policy::kSobolTable)
        if (pl.gen.sobol_staged)
          dbgz::sobol_stage_block(sob, P.gen.V, P.gen.ushift + k * (P.d - 1),
                                  (uint64_t)(P.gen.sobol_first + pl.gen.gen_base + (j - r)), pl.sobol_l0(i0),
                                  Policy::kSobolDir, P.d - 2, nb, r);
      __syncthreads();
#pragma unroll 1
      for (int li = 0; li < nb; ++li) {
        const int64_t i = i0 + li;
        if (P.ck_save == 1 && i > 0 && i % P.ck_seg == 0) {
          const int64_t slot = i / P.ck_seg - 1;
          ck_store(P.ck_ring + slot * (int64_t)W * P.ck_N, P.ck_state + slot * 4 * P.ck_N);
        }
        uint32_t xs = 0u;
        if constexpr (Policy::kSobolTable)
          if (pl.gen.sobol_staged) xs = sob_lane.at(sob, li);
        const T y = pl.emit(sg, li, i, xs);
        yr[wslot * TS + r] = y;
        wslot = wslot + 1 == W ? 0 : wslot + 1;
        T s = T(0);
        const int q0 = scol[li], q1 = scol[li + 1];
        if (staged) {
          if (sizeof(T) == 4) {
            // 4 independent partial sums: the chain of up to `bandwidth`
            // dependent FMAs becomes 4 chains a quarter as long
            T s1 = T(0), s2 = T(0), s3 = T(0);
            int q = q0;
            const T *yrr = yr + r;
            if (kPairs) {
              for (; q + 4 <= q1; q += 4) {
                const SlotVal<T> e0 = sent[q], e1 = sent[q + 1], e2 = sent[q + 2], e3 = sent[q + 3];
                s = fma(yrr[e0.off], e0.val, s);
                s1 = fma(yrr[e1.off], e1.val, s1);
                s2 = fma(yrr[e2.off], e2.val, s2);
                s3 = fma(yrr[e3.off], e3.val, s3);
              }
              for (; q < q1; ++q) s = fma(yrr[sent[q].off], sent[q].val, s);
            } else {
              for (; q + 4 <= q1; q += 4) {
                s = fma(yrr[soff[q]], sval[q], s);
                s1 = fma(yrr[soff[q + 1]], sval[q + 1], s1);
                s2 = fma(yrr[soff[q + 2]], sval[q + 2], s2);
                s3 = fma(yrr[soff[q + 3]], sval[q + 3], s3);
              }
              for (; q < q1; ++q) s = fma(yrr[soff[q]], sval[q], s);
            }
            s = (s + s1) + (s2 + s3);
          } else {
            for (int q = q0; q < q1; ++q) s = fma(yr[sent[q].off + r], sent[q].val, s);
          }
        } else {
          for (int q = q0; q < q1; ++q)
            s = fma(yr[(P.rowval[p0 + q] % W) * TS + r], P.nzval[p0 + q], s);
        }
        pl.consume(sg, s, li, i);
      }
    }
    if (P.ck_save == 2) ck_store(P.ck_ring, P.ck_state);
    if (P.tile_finish) {
      pl.tile_end(P.tgt, r, r >> 5, tile, j < P.m);
      double pv = pl.tile_value(j < P.m);
      for (int o = 16; o > 0; o >>= 1) pv += __shfl_down_sync(0xffffffffu, pv, o);
      if ((r & 31) == 0) red[r >> 5] = pv;
      __syncthreads();
      if (r == 0) P.partials[tile] = ((red[0] + red[1]) + red[2]) + red[3];
    }
  }
}

// ---- CSC of the strict upper triangle (optionally band-limited) ----------
__global__ void k_col_count(const double *U, int64_t d, int64_t band, int64_t *cnt) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= d) return;
  int64_t c = 0;
  const int64_t lo = (band > 0 && t - band > 0) ? t - band : 0;
  for (int64_t l = lo; l < t; ++l) c += U[t * d + l] != 0.0;
  cnt[t] = c;
}
__global__ void k_col_fill(const double *U, int64_t d, int64_t band, const int64_t *colptr,
                           int32_t *rowval, double *val64, float *val32, int32_t *minrow) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= d) return;
  int64_t p = colptr[t];
  int32_t mr = (int32_t)t;
  const int64_t lo = (band > 0 && t - band > 0) ? t - band : 0;
  for (int64_t l = lo; l < t; ++l) {
    const double v = U[t * d + l];
    if (v != 0.0) {
      rowval[p] = (int32_t)l;
      val64[p] = v;
      val32[p] = (float)v;
      if ((int32_t)l < mr) mr = (int32_t)l;
      ++p;
    }
  }
  minrow[t] = mr;
}

}  // namespace

// CSC of the strict upper triangle of U (d x d, column-major), limited to
// p->band super-diagonals when set; returns nnz and the bandwidth.
static int build_csc_from(dbgz_problem *p, const double *U, DevBuf &colptr_b, DevBuf &row_b, DevBuf &v64_b,
                          DevBuf &v32_b, int64_t *nnz_out, int64_t *bw_out) {
  dbgz_ctx *ctx = p->ctx;
  const int64_t d = p->d;
  std::vector<int64_t> cnt(d), colptr(d + 1);
  DBGZ_TRY(dbgz_ensure(ctx, colptr_b, sizeof(int64_t) * (d + 1)));
  k_col_count<<<(unsigned)((d + 127) / 128), 128, 0, ctx->stream>>>(U, d, p->band, (int64_t *)colptr_b.p);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(cnt.data(), colptr_b.p, sizeof(int64_t) * d, cudaMemcpyDeviceToHost,
                                     ctx->stream));
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  colptr[0] = 0;
  for (int64_t t = 0; t < d; ++t) colptr[t + 1] = colptr[t] + cnt[t];
  const int64_t nnz = colptr[d];
  *nnz_out = nnz;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(colptr_b.p, colptr.data(), sizeof(int64_t) * (d + 1), cudaMemcpyHostToDevice,
                                     ctx->stream));
  DBGZ_TRY(dbgz_ensure(ctx, row_b, sizeof(int32_t) * std::max<int64_t>(nnz, 1)));
  DBGZ_TRY(dbgz_ensure(ctx, v64_b, sizeof(double) * std::max<int64_t>(nnz, 1)));
  DBGZ_TRY(dbgz_ensure(ctx, v32_b, sizeof(float) * std::max<int64_t>(nnz, 1)));
  DevBuf minrow;
  DBGZ_TRY(dbgz_ensure(ctx, minrow, sizeof(int32_t) * d));
  k_col_fill<<<(unsigned)((d + 127) / 128), 128, 0, ctx->stream>>>(U, d, p->band, (const int64_t *)colptr_b.p,
                                                                    (int32_t *)row_b.p, (double *)v64_b.p,
                                                                    (float *)v32_b.p, (int32_t *)minrow.p);
  dbgz_count_launch(ctx);
  std::vector<int32_t> mr(d);
  cudaMemcpyAsync(mr.data(), minrow.p, sizeof(int32_t) * d, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dbgz_release(minrow);
  if (e != cudaSuccess) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "build_csc: %s", cudaGetErrorString(e));
  int64_t bw = 1;
  for (int64_t t = 1; t < d; ++t) bw = std::max<int64_t>(bw, t - mr[t]);
  *bw_out = bw;
  return DBGZ_OK;
}

int dbgz_build_csc(dbgz_problem *p) {
  int64_t nnz = 0, bw = 1;
  DBGZ_TRY(build_csc_from(p, (const double *)p->U.p, p->csc_colptr, p->csc_row, p->csc_val64, p->csc_val32, &nnz,
                          &bw));
  p->nnz = nnz;
  p->bandwidth = bw;
  return DBGZ_OK;
}

template <typename T, typename Policy>
static int launch_sparse(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  dbgz_ctx *ctx = p->ctx;
  const bool adj = pa.kind == kLoopAdjoint;
  SparseParams<T> P{};
  P.d = pa.d;
  P.nY = pa.d - 1;
  P.m = pa.m;
  P.n_reps = pa.n_reps;
  P.tiles_per_shift = (pa.m + TS - 1) / TS;
  P.n_tiles = n_tiles;
  P.tile0 = pa.tile0;
  P.gen.qmc_type = pa.qmc_type;
  P.gen.n_bits = pa.n_bits;
  P.gen.gen_base = pa.gen_base;
  P.gen.gen_base_dev = pa.gen_base_dev;
  P.gen.sobol_first = pa.sobol_first;
  // staged Sobol integers
  P.gen.sobol_staged = pa.qmc_type == DBGZ_QMC_SOBOL;
  P.gen.q = (const double *)p->q.p;
  P.gen.shift64 = (const double *)p->shifts.p;
  P.gen.shift32 = (const float *)p->shifts32.p;
  P.gen.V = (const uint32_t *)p->V.p;
  P.gen.ushift = (const uint64_t *)p->ushifts.p;
  P.colptr = (const int64_t *)(adj ? p->cscb_colptr.p : p->csc_colptr.p);
  P.rowval = (const int32_t *)(adj ? p->cscb_row.p : p->csc_row.p);
  if (sizeof(T) == 8) P.nzval = (const T *)(adj ? p->cscb_val64.p : p->csc_val64.p);
  else P.nzval = (const T *)(adj ? p->cscb_val32.p : p->csc_val32.p);
  P.tgt = sizeof(T) == 8 ? (const typename TgtT<T>::type *)p->tgt64.p : (const typename TgtT<T>::type *)p->tgt32.p;
  P.c1 = pa.c1;
  P.dc1 = pa.dc1;
  P.up1 = 1.0 - pa.c1 - pa.dc1;
  P.partials = partials;
  P.io.N = pa.grad.N;
  P.io.rows = pa.d;
  P.io.y = (T *)pa.grad.y;
  P.io.s = (T *)pa.grad.s;
  P.io.dc = (T *)pa.grad.dc;
  P.io.sbar = (T *)pa.grad.sbar;
  P.io.p = pa.grad.p;
  P.io.ga = pa.grad.ga;
  P.io.gb = pa.grad.gb;
  P.io.gu = pa.grad.gu;
  P.io.dc1 = pa.grad.dc1;
  P.io.tile0 = pa.tile0;
  P.io.row0 = pa.io_row0;
  if (pa.io_rows > 0) P.io.rows = pa.io_rows;
  P.io.store_p = pa.store_p;
  P.i_begin = pa.i_begin;
  P.i_end = pa.i_end < 0 ? P.nY : pa.i_end;
  P.ck_load = pa.ck_load;
  P.ck_save = pa.ck_save;
  P.tile_finish = pa.tile_finish;
  P.ck_in_ring = (const T *)pa.ck_in_ring;
  P.ck_in_state = pa.ck_in_state;
  P.ck_ring = (T *)pa.ck_ring;
  P.ck_state = pa.ck_state;
  P.ck_seg = pa.ck_seg > 0 ? pa.ck_seg : 1;
  P.ck_N = pa.ck_N;
  const int64_t bwid = adj ? p->bandwidth_b : p->bandwidth;
  const int W = (int)std::min<int64_t>(bwid + 1, INT32_MAX / 2);
  P.W = W;
  const int ring_cap = sizeof(T) == 8 ? 129 : 257;
  P.ring_in_smem = W <= ring_cap;
  P.max_block_nnz = (int)std::min<int64_t>(CB * std::min<int64_t>(bwid, 256), 8192);
  const size_t stage = ((sizeof(SlotVal<T>) * P.max_block_nnz + 15) & ~size_t(15)) + sizeof(int) * (CB + 4);
  const size_t smem = stage + (P.ring_in_smem ? sizeof(T) * (size_t)W * TS : 0) + 64;
  auto kern = k_genz_sparse<T, Policy>;
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  DBGZ_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TS, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t grid = std::min<int64_t>(n_tiles - pa.tile0, (int64_t)per_sm * ctx->num_sms);
  if (grid < 1) return DBGZ_OK;
  if (!P.ring_in_smem) {
    DBGZ_TRY(dbgz_ensure(ctx, p->yws, sizeof(T) * (size_t)grid * W * TS));
    P.yglob = (T *)p->yws.p;
  }
  if (pa.setup_only) return DBGZ_OK;
  kern<<<(unsigned)grid, TS, smem, ctx->stream>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

template <typename T, int GEN>
static int launch_sparse_kind(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  switch (pa.kind) {
    case kLoopForwardStore:
      if (p->lower_inf)
        return launch_sparse<T, pol::Forward<T, GEN, true, typename dbgz::StepSel<T, true>::type>>(p, pa, partials,
                                                                                               n_tiles);
      return launch_sparse<T, pol::Forward<T, GEN, true>>(p, pa, partials, n_tiles);
    case kLoopAdjoint: return launch_sparse<T, pol::Adjoint<T, GEN>>(p, pa, partials, n_tiles);
    case kLoopLogWeight:
      return launch_sparse<T, pol::Forward<T, GEN, false, typename pol::StepOf<T>::type, true>>(p, pa, partials,
                                                                                              n_tiles);
    default:
      if (p->lower_inf)
        return launch_sparse<T, pol::Forward<T, GEN, false, typename dbgz::StepSel<T, true>::type>>(
            p, pa, partials, n_tiles);
      return launch_sparse<T, pol::Forward<T, GEN, false>>(p, pa, partials, n_tiles);
  }
}

template <typename T>
static int launch_sparse_gen(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  if (pa.qmc_type == DBGZ_QMC_SOBOL) return launch_sparse_kind<T, DBGZ_QMC_SOBOL>(p, pa, partials, n_tiles);
  return launch_sparse_kind<T, DBGZ_QMC_RICHTMYER>(p, pa, partials, n_tiles);
}

int dbgz_loop_sparse(dbgz_problem *p, const PassArgs &pa, int precision, double *partials, int64_t n_tiles) {
  if (!p->csc_colptr.p) DBGZ_TRY(dbgz_build_csc(p));
  if (pa.kind == kLoopAdjoint && !p->cscb_colptr.p) {
    if (!p->Ub.p) DBGZ_TRY(dbgz_make_Ub(p));
    int64_t nnz = 0, bw = 1;
    DBGZ_TRY(build_csc_from(p, (const double *)p->Ub.p, p->cscb_colptr, p->cscb_row, p->cscb_val64, p->cscb_val32,
                            &nnz, &bw));
    p->bandwidth_b = bw;
  }
  if (precision == DBGZ_PREC_FP64) return launch_sparse_gen<double>(p, pa, partials, n_tiles);
  return launch_sparse_gen<float>(p, pa, partials, n_tiles);
}

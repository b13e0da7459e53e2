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
// y history a sample needs is the last W values (W = the factor's
// bandwidth rounded up to a power of two); it lives in a shared-memory ring
// buffer [W][128] when W fits (W <= 256 in FP32, 128 in FP64) and otherwise
// in a per-CTA slot of global memory.  The CSC entries of 32 columns are
// staged in shared memory per block of 32 dimensions.
#include "internal.cuh"
#include "genz_step.cuh"
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
  int W;                   // ring size (power of two)
  int ring_in_smem;
  int max_block_nnz;       // staging capacity (entries)
};

template <typename T>
__device__ __forceinline__ T shift_of(const dbgz::GenParams &g, int64_t idx);
template <>
__device__ __forceinline__ double shift_of<double>(const dbgz::GenParams &g, int64_t idx) {
  return g.shift64 ? g.shift64[idx] : 0.0;
}
template <>
__device__ __forceinline__ float shift_of<float>(const dbgz::GenParams &g, int64_t idx) {
  return g.shift32 ? g.shift32[idx] : 0.0f;
}

template <typename T, typename Step, int GEN>
__global__ void __launch_bounds__(TS) k_genz_sparse(const SparseParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // layout: [staged rowval int32 x cap][staged nzval T x cap][colptr of block (CB+1)][ring]
  int32_t *srow = reinterpret_cast<int32_t *>(smem_raw);
  T *sval = reinterpret_cast<T *>(smem_raw + ((sizeof(int32_t) * P.max_block_nnz + 15) & ~size_t(15)));
  int *scol = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(sval) +
                                      ((sizeof(T) * P.max_block_nnz + 15) & ~size_t(15)));
  double *sq = reinterpret_cast<double *>(scol + CB + 2 + 2);
  T *ssh = reinterpret_cast<T *>(sq + CB);
  typename TgtT<T>::type *stg =
      reinterpret_cast<typename TgtT<T>::type *>(reinterpret_cast<unsigned char *>(ssh) + 16 * ((sizeof(T) * CB + 15) / 16));
  T *ring = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(stg) + sizeof(*stg) * CB);
  __shared__ double red[TS / 32];
  const int r = threadIdx.x;
  const int Wm = P.W - 1;
  T *yr = P.ring_in_smem ? ring : P.yglob + (int64_t)blockIdx.x * P.W * TS;
  dbgz::GenParams gen = P.gen;
  gen.qmc_type = GEN;

  for (int64_t tile = blockIdx.x; tile < P.n_tiles; tile += gridDim.x) {
    const int64_t k = tile / P.tiles_per_shift;
    const int64_t j = (tile - k * P.tiles_per_shift) * TS + r;
    Step st;
    st.init(P.c1, P.dc1, P.up1);
    for (int64_t i0 = 0; i0 < P.nY; i0 += CB) {
      const int nb = (int)(P.nY - i0 < CB ? P.nY - i0 : CB);
      // stage the CSC columns i0+1 .. i0+nb (targets of y-indices i0..i0+nb-1)
      __syncthreads();
      const int64_t p0 = P.colptr[i0 + 1], p1 = P.colptr[i0 + nb + 1];
      const int cnt = (int)(p1 - p0);
      const bool staged = cnt <= P.max_block_nnz;
      if (staged)
        for (int e = r; e < cnt; e += TS) {
          srow[e] = P.rowval[p0 + e];
          sval[e] = P.nzval[p0 + e];
        }
      if (r <= nb) scol[r] = (int)(P.colptr[i0 + 1 + r] - p0);
      if (r < nb) {
        sq[r] = gen.q ? gen.q[i0 + r] : 0.0;
        ssh[r] = shift_of<T>(gen, k * P.nY + i0 + r);
        stg[r] = P.tgt[i0 + r + 1];
      }
      __syncthreads();
#pragma unroll 1
      for (int li = 0; li < nb; ++li) {
        const int64_t i = i0 + li;
        T y = st.quantile(gen, P.d, j, k, i, sq[li], ssh[li]);
        yr[(i & Wm) * TS + r] = y;
        T s = T(0);
        const int q0 = scol[li], q1 = scol[li + 1];
        if (staged) {
          for (int q = q0; q < q1; ++q) s = fma(yr[(srow[q] & Wm) * TS + r], sval[q], s);
        } else {
          for (int q = q0; q < q1; ++q)
            s = fma(yr[(P.rowval[p0 + q] & Wm) * TS + r], P.nzval[p0 + q], s);
        }
        const auto tg = stg[li];
        st.cdf(s, tg.a, tg.b, tg.inv_u, 0);
      }
    }
    double pv = (j < P.m) ? st.p : 0.0;
    for (int o = 16; o > 0; o >>= 1) pv += __shfl_down_sync(0xffffffffu, pv, o);
    if ((r & 31) == 0) red[r >> 5] = pv;
    __syncthreads();
    if (r == 0) P.partials[tile] = ((red[0] + red[1]) + red[2]) + red[3];
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

int dbgz_build_csc(dbgz_problem *p) {
  dbgz_ctx *ctx = p->ctx;
  const int64_t d = p->d;
  std::vector<int64_t> cnt(d), colptr(d + 1);
  DBGZ_TRY(dbgz_ensure(ctx, p->csc_colptr, sizeof(int64_t) * (d + 1)));
  k_col_count<<<(unsigned)((d + 127) / 128), 128, 0, ctx->stream>>>((const double *)p->U.p, d, p->band,
                                                                     (int64_t *)p->csc_colptr.p);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(cnt.data(), p->csc_colptr.p, sizeof(int64_t) * d, cudaMemcpyDeviceToHost,
                                     ctx->stream));
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  colptr[0] = 0;
  for (int64_t t = 0; t < d; ++t) colptr[t + 1] = colptr[t] + cnt[t];
  const int64_t nnz = colptr[d];
  p->nnz = nnz;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(p->csc_colptr.p, colptr.data(), sizeof(int64_t) * (d + 1),
                                     cudaMemcpyHostToDevice, ctx->stream));
  DBGZ_TRY(dbgz_ensure(ctx, p->csc_row, sizeof(int32_t) * std::max<int64_t>(nnz, 1)));
  DBGZ_TRY(dbgz_ensure(ctx, p->csc_val64, sizeof(double) * std::max<int64_t>(nnz, 1)));
  DBGZ_TRY(dbgz_ensure(ctx, p->csc_val32, sizeof(float) * std::max<int64_t>(nnz, 1)));
  DevBuf minrow;
  DBGZ_TRY(dbgz_ensure(ctx, minrow, sizeof(int32_t) * d));
  k_col_fill<<<(unsigned)((d + 127) / 128), 128, 0, ctx->stream>>>(
      (const double *)p->U.p, d, p->band, (const int64_t *)p->csc_colptr.p, (int32_t *)p->csc_row.p,
      (double *)p->csc_val64.p, (float *)p->csc_val32.p, (int32_t *)minrow.p);
  dbgz_count_launch(ctx);
  std::vector<int32_t> mr(d);
  cudaMemcpyAsync(mr.data(), minrow.p, sizeof(int32_t) * d, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dbgz_release(minrow);
  if (e != cudaSuccess) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "build_csc: %s", cudaGetErrorString(e));
  int64_t bw = 1;
  for (int64_t t = 1; t < d; ++t) bw = std::max<int64_t>(bw, t - mr[t]);
  p->bandwidth = bw;
  return DBGZ_OK;
}

template <typename T, typename Step>
static int launch_sparse(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  dbgz_ctx *ctx = p->ctx;
  SparseParams<T> P{};
  P.d = pa.d;
  P.nY = pa.d - 1;
  P.m = pa.m;
  P.n_reps = pa.n_reps;
  P.tiles_per_shift = (pa.m + TS - 1) / TS;
  P.n_tiles = n_tiles;
  P.gen.qmc_type = pa.qmc_type;
  P.gen.n_bits = pa.n_bits;
  P.gen.gen_base = pa.gen_base;
  P.gen.sobol_first = pa.sobol_first;
  P.gen.q = (const double *)p->q.p;
  P.gen.shift64 = (const double *)p->shifts.p;
  P.gen.shift32 = (const float *)p->shifts32.p;
  P.gen.V = (const uint32_t *)p->V.p;
  P.gen.ushift = (const uint64_t *)p->ushifts.p;
  P.colptr = (const int64_t *)p->csc_colptr.p;
  P.rowval = (const int32_t *)p->csc_row.p;
  P.nzval = sizeof(T) == 8 ? (const T *)p->csc_val64.p : (const T *)p->csc_val32.p;
  P.tgt = sizeof(T) == 8 ? (const typename TgtT<T>::type *)p->tgt64.p : (const typename TgtT<T>::type *)p->tgt32.p;
  P.c1 = pa.c1;
  P.dc1 = pa.dc1;
  P.up1 = 1.0 - pa.c1 - pa.dc1;
  P.partials = partials;
  int W = 1;
  while (W < p->bandwidth + 1) W <<= 1;
  P.W = W;
  const int ring_cap = sizeof(T) == 8 ? 128 : 256;
  P.ring_in_smem = W <= ring_cap;
  P.max_block_nnz = (int)std::min<int64_t>(CB * std::min<int64_t>(p->bandwidth, 256), 8192);
  const size_t stage = ((sizeof(int32_t) * P.max_block_nnz + 15) & ~size_t(15)) +
                       ((sizeof(T) * P.max_block_nnz + 15) & ~size_t(15)) + sizeof(int) * (CB + 4) +
                       sizeof(double) * CB + 16 * ((sizeof(T) * CB + 15) / 16) +
                       sizeof(typename TgtT<T>::type) * CB;
  const size_t smem = stage + (P.ring_in_smem ? sizeof(T) * (size_t)W * TS : 0) + 64;
  auto kern = pa.qmc_type == DBGZ_QMC_SOBOL ? k_genz_sparse<T, Step, DBGZ_QMC_SOBOL>
                                             : k_genz_sparse<T, Step, DBGZ_QMC_RICHTMYER>;
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  DBGZ_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TS, smem));
  per_sm = std::max(per_sm, 1);
  const int64_t grid = std::min<int64_t>(n_tiles, (int64_t)per_sm * ctx->num_sms);
  if (!P.ring_in_smem) {
    DBGZ_TRY(dbgz_ensure(ctx, p->yws, sizeof(T) * (size_t)grid * W * TS));
    P.yglob = (T *)p->yws.p;
  }
  kern<<<(unsigned)grid, TS, smem, ctx->stream>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_loop_sparse(dbgz_problem *p, const PassArgs &pa, int precision, double *partials, int64_t n_tiles) {
  if (!p->csc_colptr.p) DBGZ_TRY(dbgz_build_csc(p));
  if (precision == DBGZ_PREC_FP64) return launch_sparse<double, dbgz::StepFp64>(p, pa, partials, n_tiles);
  return launch_sparse<float, dbgz::StepFp32>(p, pa, partials, n_tiles);
}

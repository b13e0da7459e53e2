// loop_simt_kernels.cuh -- device code of the SIMT integration loop (see
// loop_simt.cu for the decomposition).  Kept in a header so that every
// launcher instantiates the same kernel templates.
#pragma once
#include "internal.cuh"
#include "genz_step.cuh"
#include "policies.cuh"

namespace simt {

constexpr int TS = 128;   // samples per tile
constexpr int G = 64;     // y-indices per group
constexpr int SB = 32;    // y-indices per sequential sub-block
constexpr int KC = 16;    // K chunk of the group GEMM
constexpr int NT = 256;   // threads per CTA

template <typename T>
struct TgtOf;
template <>
struct TgtOf<double> {
  using type = TargetParams64;
};
template <>
struct TgtOf<float> {
  using type = TargetParams32;
};

template <typename T>
struct SimtParams {
  int64_t d, m, n_reps, tiles_per_shift, n_tiles, Dp;
  int64_t tile0;  // tiles [tile0, n_tiles) of the pass
  dbgz::GenParams gen;
  const T *U;  // d x d col-major coefficient array (policies.cuh)
  const typename TgtOf<T>::type *tgt;
  double c1, dc1, up1;
  int cdf_form;
  T *yws;            // gridDim.x slots of Dp x TS
  double *partials;  // n_tiles
  pol::GradIO<T> io;
};

template <typename T>
struct SimtSmem {
  T Ss[G][TS];                // group partial sums, [target][sample]
  union {
    struct {
      T Ys[KC][TS];
      T Us[KC][G + 4];
    } gemm;
    T Ysub[SB][TS];           // emitted values of the last sub-block
  } u;
  T Ublk[SB][SB + 1];         // coefficients of the sub-block (and of the cross block)
  pol::Staged<T> sg;
  uint32_t sob[SB][dbgz::kSobolRow];  // Sobol integers of the sub-block (dbgz::sobol_stage_block)
  double red[NT / 32];
};

// One tile of 128 samples of the problem P (all NT threads of the CTA; Yw
// is the CTA's slot of the Y workspace).
// Policy: pol::Forward<...> or pol::Adjoint<...> (policies.cuh).
template <typename T, typename Policy>
__device__ __forceinline__ void simt_tile(const SimtParams<T> &P, SimtSmem<T> &sm, T *Yw, int64_t tile) {
  const int tid = threadIdx.x;
  const int64_t d = P.d, nY = d - 1;
  const int64_t last_g0 = ((nY - 1) / G) * G;  // start of the last group
  {
    const int r = tid;  // sample row for the scalar threads (tid < TS)
    const int64_t k = tile / P.tiles_per_shift;
    const int64_t j = (tile - k * P.tiles_per_shift) * TS + r;
    Policy pl;
    if (tid < TS) pl.tile_begin(P.gen, d, tile, P.tiles_per_shift, r, P.c1, P.dc1, P.up1, P.cdf_form, P.io);
    // this row's terms of the staged Sobol integers of the tile
    const dbgz::SobolLane sob_lane(r, tid < TS ? (uint64_t)(P.gen.sobol_first + pl.gen.gen_base + (j - r)) : 0u);

    for (int64_t g0 = 0; g0 < nY; g0 += G) {
      const int ng = (int)(nY - g0 < (int64_t)G ? nY - g0 : (int64_t)G);
      // ---- group GEMM: Ss[t][r] = sum_{l<g0} V[l][r] C[l][g0+t] ----
      {
        const int tx = tid & 15, ty = tid >> 4;
        T acc[8][4];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
        for (int64_t l0 = 0; l0 < g0; l0 += KC) {
#pragma unroll
          for (int e = 0; e < KC * TS / NT; ++e) {
            int idx = tid + e * NT;
            int kk = idx / TS, rr = idx % TS;
            sm.u.gemm.Ys[kk][rr] = Yw[(l0 + kk) * TS + rr];
          }
#pragma unroll
          for (int e = 0; e < KC * G / NT; ++e) {
            int idx = tid + e * NT;
            int t = idx / KC, kk = idx % KC;
            int64_t tgt = g0 + 1 + t;
            sm.u.gemm.Us[kk][t] = tgt < d ? P.U[tgt * d + l0 + kk] : T(0);
          }
          __syncthreads();
#pragma unroll
          for (int kk = 0; kk < KC; ++kk) {
            T av[8], bv[4];
#pragma unroll
            for (int a = 0; a < 8; ++a) av[a] = sm.u.gemm.Ys[kk][ty * 8 + a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = sm.u.gemm.Us[kk][tx * 4 + b];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
          }
          __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) sm.Ss[tx * 4 + b][ty * 8 + a] = acc[a][b];
        __syncthreads();
      }
      // ---- sequential sub-blocks ----
      for (int sb = 0; sb < ng; sb += SB) {
        const int nsb = min(SB, ng - sb);
        const int64_t l_base = g0 + sb;
        for (int e = tid; e < SB * SB; e += NT) {
          int li = e % SB, ti = e / SB;
          int64_t l = l_base + li, t = l_base + ti + 1;
          sm.Ublk[li][ti] = (li <= ti && li < nsb && ti < nsb) ? P.U[t * d + l] : T(0);
        }
        if (tid < TS) {
          pl.stage(sm.sg, P.tgt, tid, l_base, nsb);
          if constexpr (Policy::kSobolTable)
            if (pl.gen.sobol_staged)
              dbgz::sobol_stage_block(sm.sob, P.gen.V, P.gen.ushift + k * (d - 1),
                                      (uint64_t)(P.gen.sobol_first + pl.gen.gen_base + (j - r)),
                                      pl.sobol_l0(l_base), Policy::kSobolDir, d - 2, nsb, r);
        }
        __syncthreads();
        if (tid < TS) {
          // in-block dot in the reference's order (src/qmc.jl:394-403):
          // acc = S[target] + v_{l_base} C[..] + ... + v_l C[l, l]
#pragma unroll 1
          for (int li = 0; li < nsb; ++li) {
            const int64_t l = l_base + li;
            uint32_t xs = 0u;
            if constexpr (Policy::kSobolTable)
              if (pl.gen.sobol_staged) xs = sob_lane.at(sm.sob, li);
            T v = pl.emit(sm.sg, li, l, xs);
            sm.u.Ysub[li][r] = v;
            if (g0 < last_g0) Yw[l * TS + r] = v;
            T acc = sm.Ss[sb + li][r];
#pragma unroll 4
            for (int mi = 0; mi <= li; ++mi) acc = fma(sm.u.Ysub[mi][r], sm.Ublk[mi][li], acc);
            pl.consume(sm.sg, acc, li, l);
          }
        }
        __syncthreads();
        // cross update: Ss[sb+SB+t][r] += sum_li Ysub[li][r] C[l_base+li][l_base+SB+t]
        if (sb + SB < ng) {
          const int nt2 = min(SB, ng - sb - SB);
          for (int e = tid; e < SB * SB; e += NT) {
            int li = e % SB, ti = e / SB;
            int64_t t = l_base + SB + ti + 1;
            sm.Ublk[li][ti] = (ti < nt2) ? P.U[t * d + l_base + li] : T(0);
          }
          __syncthreads();
          const int rr = tid & (TS - 1), half = tid / TS;  // 2 threads per sample
#pragma unroll 4
          for (int ti = half * 16; ti < half * 16 + 16; ++ti) {
            T acc = sm.Ss[sb + SB + ti][rr];
#pragma unroll
            for (int li = 0; li < SB; ++li) acc = fma(sm.u.Ysub[li][rr], sm.Ublk[li][ti], acc);
            sm.Ss[sb + SB + ti][rr] = acc;
          }
          __syncthreads();
        }
      }
    }
    // ---- per-tile end and sum of p (fixed order) ----
    if (tid < TS) pl.tile_end(P.tgt, tid, 0, tile, j < P.m);
    double pv = (tid < TS) ? pl.tile_value(j < P.m) : 0.0;
    for (int o = 16; o > 0; o >>= 1) pv += __shfl_down_sync(0xffffffffu, pv, o);
    if ((tid & 31) == 0) sm.red[tid >> 5] = pv;
    __syncthreads();
    if (tid == 0) {
      double sum = 0.0;
      for (int w = 0; w < NT / 32; ++w) sum += sm.red[w];
      P.partials[tile] = sum;
    }
    __syncthreads();
  }
}

template <typename T, typename Policy>
__global__ void __launch_bounds__(NT, 2) k_genz_simt(SimtParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimtSmem<T> &sm = *reinterpret_cast<SimtSmem<T> *>(smem_raw);
  T *Yw = P.yws + (int64_t)blockIdx.x * P.Dp * TS;
  for (int64_t tile = P.tile0 + blockIdx.x; tile < P.n_tiles; tile += gridDim.x)
    simt_tile<T, Policy>(P, sm, Yw, tile);
}

// Many problems in one launch: a work item is a run of tiles of one problem
// (items ordered largest problem first); persistent CTAs take items from a
// global counter.  Each problem's parameters (pointers into packed arrays,
// its own first-dimension constants) are copied to shared memory per item;
// the Y workspace slots are sized for the largest problem (Dp).
struct BatchItem {
  int32_t prob, tile0, ntiles, pad;
};

template <typename T, typename Policy>
__global__ void __launch_bounds__(NT, 2) k_genz_simt_batch(const SimtParams<T> *params, const BatchItem *items,
                                                           int64_t n_items, unsigned long long *counter, T *yws,
                                                           int64_t Dp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimtSmem<T> &sm = *reinterpret_cast<SimtSmem<T> *>(smem_raw);
  __shared__ SimtParams<T> Ps;
  __shared__ long long cur;
  T *Yw = yws + (int64_t)blockIdx.x * Dp * TS;
  for (;;) {
    if (threadIdx.x == 0) {
      cur = (long long)atomicAdd(counter, 1ull);
      if (cur < n_items) Ps = params[items[cur].prob];
    }
    __syncthreads();
    const long long it = cur;
    if (it >= n_items) break;
    const BatchItem bi = items[it];
    for (int64_t tile = bi.tile0; tile < (int64_t)bi.tile0 + bi.ntiles; ++tile) simt_tile<T, Policy>(Ps, sm, Yw, tile);
    __syncthreads();
  }
}

// Per shift: Neumaier-compensated sum of its tile sums in tile order, then
// the running mean of src/qmc.jl:437-442.
static __global__ void k_finalize(const double *partials, int64_t tiles_per_shift, int64_t n_reps,
                           int64_t n_pts0, int64_t m, double *reps) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n_reps) return;
  const double *pk = partials + k * tiles_per_shift;
  double s = 0.0, c = 0.0;
  for (int64_t t = 0; t < tiles_per_shift; ++t) {
    double x = pk[t];
    double tt = s + x;
    if (fabs(s) >= fabs(x)) c += (s - tt) + x;
    else c += (x - tt) + s;
    s = tt;
  }
  s += c;
  double inv_tot = 1.0 / (double)(n_pts0 + m);
  double mean_rep = s * inv_tot;
  double old_weight = (double)n_pts0 * inv_tot;
  reps[k] = fma(reps[k], old_weight, mean_rep);
}

}  // namespace simt

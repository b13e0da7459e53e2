// policies.cuh -- what one sequential step of the integration loops does.
//
// Both loop kernels (SIMT and tensor-core) walk an "emitter" index l =
// 0..d-2 in order; step l emits a value v_l, and the contraction delivers
// to step l the receiver sum r_l = sum_{l' <= l} v_{l'} C[l', l] (the
// emitter's own diagonal term included), where C is an upper-triangular
// coefficient matrix given as a d x d column-major array with C[l', l] at
// [(l + 1) * d + l'].  A policy supplies v_l (emit) and uses r_l
// (consume):
//
//  * Forward (qmc_loop!, src/qmc.jl:315-444): C = U, v_l = y_l = Phi^-1(u_l),
//    r_l = s_{l+1}, consume = the CDF update of variable l+1.  With STORE it
//    also records y_l, s_{l+1}, dc_{l+1} and p per sample for the adjoint.
//  * Adjoint (no counterpart in the reference): the reverse recurrence
//      ybar_l = sum_{t > l} sbar_t U[l, t]
//    has the same triangular shape once indices are reversed: emitter
//    l' = d-1-t, C = the anti-transpose of U (C[i, j] = U[d-1-j, d-1-i]),
//    v_{l'} = sbar_t, r_{l'} = ybar_{t-1}.  emit computes sbar_t of
//    variable t = d-1-l' from the stored forward state and the saved
//    ybar_t; consume saves ybar_{t-1} for the next step.
//
// Adjoint of one sample (L = p = prod_t dc_t; c_t = Phi(alpha_t),
// e_t = Phi(beta_t), alpha_t = (a_t - s_t)/U_tt, u_t = (1-w_t) c_t + w_t e_t,
// y_t = Phi^-1(u_t)):
//   ubar_t = ybar_t / phi(y_t)                          (0 if u_t was clamped)
//   ebar_t = p/dc_t + ubar_t w_t,   cbar_t = -p/dc_t + ubar_t (1 - w_t)
//   dL/da_t = cbar_t phi(alpha_t)/U_tt,  dL/db_t = ebar_t phi(beta_t)/U_tt
//   sbar_t = -(dL/da_t + dL/db_t),  dL/dU_tt = -(dL/da_t alpha_t + dL/db_t beta_t)
//   dL/dU[l,t] = y_l sbar_t  (l < t; accumulated over samples by a GEMM)
// The forward clamps (|x| < 9 in erf units, u in [eps64, 1-eps64]) pass no
// derivative.  Everything is linear in p, so the recurrence runs with unit
// seed (p replaced by 1) and per-sample results are scaled by p when they
// are accumulated.
#pragma once
#include <type_traits>

#include "internal.cuh"
#include "genz_step.cuh"

namespace pol {

constexpr int PB = 32;  // staged dimensions per block

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

// Per-block staging shared by every policy: target constants, lattice
// generator and shift of the block's steps (index mapping per policy).
template <typename T>
struct Staged {
  typename TgtT<T>::type tg[PB];
  double qv[PB];
  T shv[PB];
};

// Arrays of the forward state kept for the adjoint, `rows` (= d) indices per
// sample, N samples.  FP64: [index][sample] (row stride N, the layout of the
// library DGEMM of the factor gradient).  FP32: tile-major, [tile][index]
// [128 samples of the tile]: one tile's state is one contiguous block of
// d x 512 bytes, so a step's 128 values are one coalesced 512-byte row and
// the factor-gradient GEMM reads 32-sample slices of many rows from a few
// pages (with row stride N = 2^21 samples every row lies on its own page of
// the GPU's address translation; this layout took the d = 1000 gradient from
// 92 to 81 ms).
template <typename T>
struct GradIO {
  int64_t N = 0, rows = 0;
  T *y = nullptr;     // y_l,  l = 0..d-2
  T *s = nullptr;     // s_t,  t = 1..d-1 (row t)
  T *dc = nullptr;    // dc_t, t = 1..d-1 (row t)
  double *p = nullptr;
  T *sbar = nullptr;  // p * sbar_t, t = 1..d-1 (row t)
  double *ga = nullptr, *gb = nullptr, *gu = nullptr;  // [((tile - tile0) * 4 + warp) * d + t]
  double dc1 = 0.0;   // dc of variable 0
  int64_t tile0 = 0;  // first tile of the sample chunk these arrays hold (sample g = (tile - tile0) * 128 + r)
  // first row the arrays hold (a dimension segment's recomputed state holds
  // rows row0 .. row0 + rows - 1)
  int64_t row0 = 0;
  int store_p = 0;    // a forward pass without stored state still writes p (checkpointed gradients)
  __device__ __forceinline__ int64_t at(int64_t row, int64_t g) const {
    if (sizeof(T) == 4) return ((g >> 7) * rows + (row - row0)) * 128 + (g & 127);
    return (row - row0) * N + g;
  }
  // at(row, g) = at0(g) + row * stride(): the sample's part, computed once per
  // tile, and a row stride (a constant 128 for FP32), so that a step's
  // address is one multiply-add on the row (constant offsets inside a chunk)
  __device__ __forceinline__ int64_t at0(int64_t g) const {
    if (sizeof(T) == 4) return ((g >> 7) * rows - row0) * 128 + (g & 127);
    return g - row0 * N;
  }
  __device__ __forceinline__ int64_t stride() const { return sizeof(T) == 4 ? (int64_t)128 : N; }
};

// Asynchronous global -> shared copy of `BYTES` (4, 8 or 16) bytes, or zeros
// when !valid (no bytes are read then; `src` must still be a mapped address).
template <int BYTES>
__device__ __forceinline__ void cp_async_or_zero(void *dst_smem, const void *src, bool valid) {
  const uint32_t dst = (uint32_t)__cvta_generic_to_shared(dst_smem);
  const int n = valid ? BYTES : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(dst), "l"(src), "n"(BYTES), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ T shift_at(const dbgz::GenParams &g, int64_t idx);
template <>
__device__ __forceinline__ double shift_at<double>(const dbgz::GenParams &g, int64_t idx) {
  return g.shift64 ? g.shift64[idx] : 0.0;
}
template <>
__device__ __forceinline__ float shift_at<float>(const dbgz::GenParams &g, int64_t idx) {
  return g.shift32 ? g.shift32[idx] : 0.0f;
}

// Step numerics by working type.
template <typename T>
struct StepOf;
template <>
struct StepOf<double> {
  using type = dbgz::StepFp64;
};
template <>
struct StepOf<float> {
  using type = dbgz::StepFp32;
};

// ---------------------------------------------------------------- forward ---
// LOGW: also sum log dc over the sample's variables and write the sum (the
// sample's log-weight) to io.p at the tile's end (kLoopLogWeight)
template <typename T, int GEN, bool STORE, typename Step = typename StepOf<T>::type, bool LOGW = false>
struct Forward {
  static constexpr bool kPlain = !STORE;  // a forward pass that keeps no state
  // consume_deferred + tail_repair available (the FP32 steps): the loop may
  // run a chunk of steps without the same-tail branch
  static constexpr bool kDeferTail = std::is_same<T, float>::value;
  // takes staged Sobol integers (GenParams::sobol_staged); not in the pass
  // that keeps the state for the adjoint (measured on the banded d = 10^4,
  // bandwidth 64 workload at 2^14 x 10 Sobol points:
  // the gradient call 125.1 ms without, 136.9 ms with them)
  static constexpr bool kSobolTable = GEN == DBGZ_QMC_SOBOL && !STORE;
  // the QMC dimension of step li of a block: lbase + li
  static constexpr int kSobolDir = 1;
  __device__ __forceinline__ int64_t sobol_l0(int64_t lbase) const { return lbase; }
  Step st;
  double lw;  // LOGW: log of the weight so far
  uint32_t rmask;  // steps k of the current chunk whose weight factor consume_deferred left out
  dbgz::GenParams gen;
  int64_t j, k, g;  // point index in the pass, shift, global sample index
  int64_t ga0;      // io.at0(g)
  int64_t d;
  int cdf_form;
  GradIO<T> io;

  __device__ __forceinline__ void tile_begin(const dbgz::GenParams &gp, int64_t d_, int64_t tile,
                                             int64_t tiles_per_shift, int r, double c1, double dc1,
                                             double up1, int cdf_form_, const GradIO<T> &io_) {
    gen = gp;
    gen.qmc_type = GEN;
    if (!kSobolTable) gen.sobol_staged = 0;  // points from sobol_warp whatever the launch says
    if (gp.gen_base_dev) gen.gen_base = *gp.gen_base_dev;
    d = d_;
    k = tile / tiles_per_shift;
    j = (tile - k * tiles_per_shift) * 128 + r;
    g = (tile - io_.tile0) * 128 + r;
    cdf_form = cdf_form_;
    io = io_;
    ga0 = io.at0(g);
    st.init(c1, dc1, up1);
    st.set_form(cdf_form_);
    if (LOGW) lw = log(dc1);
    rmask = 0u;
  }
  // cooperative: r in [0, 128)
  __device__ __forceinline__ void stage(Staged<T> &sg, const typename TgtT<T>::type *tgt, int r,
                                        int64_t lbase, int nval) const {
    if (r < nval) {
      sg.tg[r] = tgt[lbase + r + 1];
      sg.qv[r] = gen.q ? gen.q[lbase + r] : 0.0;
      sg.shv[r] = shift_at<T>(gen, k * (d - 1) + lbase + r);
    }
  }
  // stage() by asynchronous copies (FP32 staging only): the caller commits
  // and waits
  __device__ __forceinline__ void stage_async(Staged<T> &sg, const typename TgtT<T>::type *tgt, int r,
                                              int64_t lbase, int nval) const {
    static_assert(sizeof(typename TgtT<T>::type) == 16 && sizeof(T) == 4, "FP32 staging");
    if (r < nval) {
      const int64_t si = k * (d - 1) + lbase + r;
      cp_async_or_zero<16>(&sg.tg[r], &tgt[lbase + r + 1], true);
      cp_async_or_zero<8>(&sg.qv[r], gen.q ? (const void *)(gen.q + lbase + r) : (const void *)tgt, gen.q != nullptr);
      cp_async_or_zero<4>(&sg.shv[r], gen.shift32 ? (const void *)(gen.shift32 + si) : (const void *)tgt,
                          gen.shift32 != nullptr);
    }
  }
  // xs: the Sobol integer of this point in dimension l when the loop stages
  // them (GenParams::sobol_staged), else unused
  __device__ __forceinline__ T emit(const Staged<T> &sg, int li, int64_t l, uint32_t xs = 0u) {
    const T y = st.template quantile<!STORE>(gen, d, j, k, l, sg.qv[li], sg.shv[li], xs);
    if (STORE) __stcs(io.y + ga0 + l * io.stride(), y);
    return y;
  }
  // chunked form (8 steps whose per-sample inputs may be loaded up front)
  __device__ __forceinline__ void chunk_begin(int64_t, int) {}
  __device__ __forceinline__ void chunk_end(int64_t, int) {}
  __device__ __forceinline__ T emit_k(const Staged<T> &sg, int li, int64_t l, int, uint32_t xs) {
    return emit(sg, li, l, xs);
  }
  __device__ __forceinline__ T emit_k_fast(const Staged<T> &sg, int li, int64_t l, int k, uint32_t xs) {
    return emit_k(sg, li, l, k, xs);
  }
  __device__ __forceinline__ void consume(const Staged<T> &sg, T s, int li, int64_t l) {
    const auto tg = sg.tg[li];
    st.cdf(s, tg.a, tg.b, tg.inv_u, cdf_form);
    if (LOGW) lw += log((double)st.dc);
    if (STORE) {
      __stcs(io.s + ga0 + (l + 1) * io.stride(), s);
      __stcs(io.dc + ga0 + (l + 1) * io.stride(), (T)st.dc);
    }
  }
  // consume for step k (0..7) of a chunk, without the same-tail branch
  // (Step::cdf_deferred): a factor left out is recorded in rmask and
  // multiplied in by tail_repair at the chunk's end
  __device__ __forceinline__ void consume_deferred(const Staged<T> &sg, T s, int li, int64_t l, int k) {
    const auto tg = sg.tg[li];
    const bool left = st.cdf_deferred(s, tg.a, tg.b, tg.inv_u);
    rmask |= left ? (1u << k) : 0u;
    if (LOGW) lw += left ? 0.0 : log((double)st.dc);
    if (STORE) {
      __stcs(io.s + ga0 + (l + 1) * io.stride(), s);
      __stcs(io.dc + ga0 + (l + 1) * io.stride(), (T)st.dc);
    }
  }
  // The factors consume_deferred left out in a chunk of 8 steps starting at
  // staged index li0 (y-index l0), from the same sums s[0..7] (the chunk's
  // consumed values, still in place): one warp-uniform branch per chunk,
  // taken only when some sample of the warp had such a step.  The weight
  // then has the same factors as with cdf, the FP64 products in another order.
  template <int N>
  __device__ __forceinline__ void tail_repair(const Staged<T> &sg, const T (&s)[N], int li0, int64_t l0) {
    if (__any_sync(0xffffffffu, rmask != 0u)) {
      // one call site: the step's sum picked by selects (a dynamic index
      // would put s[] in local memory)
      for (uint32_t m = rmask; m != 0u; m &= m - 1u) {
        const int k = __ffs((int)m) - 1;
        T sk = s[0];
#pragma unroll
        for (int kk = 1; kk < 8; ++kk) sk = k == kk ? s[kk] : sk;
        const auto tg = sg.tg[li0 + k];
        const float d = Step::tail_exact(sk, tg.a, tg.b, tg.inv_u);
        st.p *= (double)d;
        if (LOGW) lw += log((double)d);
        if (STORE) __stcs(io.dc + ga0 + (l0 + k + 1) * io.stride(), (T)d);
      }
      rmask = 0u;
    }
  }
  // value of this sample added to the tile's sum of p
  __device__ __forceinline__ double tile_value(bool valid) {
    if (STORE || io.store_p) io.p[g] = valid ? st.p : 0.0;
    if (LOGW) io.p[g] = valid ? lw : -INFINITY;
    return valid ? st.p : 0.0;
  }
  __device__ __forceinline__ void tile_end(const typename TgtT<T>::type *, int, int, int64_t, bool) {}
  // the recursion's state between two steps (checkpoints of the banded gradient)
  __device__ __forceinline__ void pack(double (&v)[4]) const { st.pack(v); }
  __device__ __forceinline__ void unpack(const double (&v)[4]) { st.unpack(v); }
};

// x rounded to the nearest TF32 value (low 13 mantissa bits zero)
__device__ __forceinline__ float tf32_rn(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// ---------------------------------------------------------------- adjoint ---
template <typename T, int GEN>
struct Adjoint {
  static constexpr bool kPlain = false;
  static constexpr bool kDeferTail = false;
  // the loop may run a chunk with emit_k_fast (no per-step vote) and redo it
  // with emit_k when some lane's FP32 terms left FP32 range (bad)
  static constexpr bool kChunkRedo = sizeof(T) == 4;
  bool bad;
  // takes staged Sobol integers (GenParams::sobol_staged) where the loop
  // stages them; the QMC dimension of step li of a block: d - 1 - lbase - li
  static constexpr bool kSobolTable = GEN == DBGZ_QMC_SOBOL;
  static constexpr int kSobolDir = -1;
  __device__ __forceinline__ int64_t sobol_l0(int64_t lbase) const { return d - 1 - lbase; }
  dbgz::GenParams gen;
  int64_t j, k, g, d, tile;
  double jd;    // gen.gen_base + j + 1: the lattice point's multiplier
  int64_t ga0;  // io.at0(g)
  GradIO<T> io;
  // saved receiver value: ybar of the variable the next step handles, in the
  // working type (it is a sum of the loop's working type; no round trip
  // through FP64 on the FP32 chain)
  T ybar;
  double p;     // this sample's weight (the seed scale)
  // FP32 paths: the warp's largest weight, and this sample's weight relative
  // to it (in [0, 1]); the per-variable sums over the warp's samples are then
  // taken in FP32 and scaled back by wmax in FP64
  double wmax;
  float wrel;
  int warp, lane;

  __device__ __forceinline__ void tile_begin(const dbgz::GenParams &gp, int64_t d_, int64_t tile_,
                                             int64_t tiles_per_shift, int r, double, double, double, int,
                                             const GradIO<T> &io_) {
    gen = gp;
    gen.qmc_type = GEN;
    if (!kSobolTable) gen.sobol_staged = 0;
    if (gp.gen_base_dev) gen.gen_base = *gp.gen_base_dev;
    d = d_;
    tile = tile_;
    k = tile / tiles_per_shift;
    j = (tile - k * tiles_per_shift) * 128 + r;
    jd = (double)(gen.gen_base + j + 1);
    g = (tile - io_.tile0) * 128 + r;
    io = io_;
    ga0 = io.at0(g);
    ybar = T(0);  // variable d-1 has no u: nothing downstream of it
    p = io.p[g];
    warp = r >> 5;
    lane = r & 31;
    if (sizeof(T) == 4) {
      double m = p;
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      wmax = m;
      wrel = m > 0.0 ? (float)(p / m) : 0.f;
    }
  }
  // step li of the block handles variable t = d-1-(lbase+li); its point is
  // QMC dimension t (y-index t), which exists for t <= d-2
  __device__ __forceinline__ void stage(Staged<T> &sg, const typename TgtT<T>::type *tgt, int r,
                                        int64_t lbase, int nval) const {
    if (r < nval) {
      const int64_t t = d - 1 - (lbase + r);
      sg.tg[r] = tgt[t];
      sg.qv[r] = (t <= d - 2 && gen.q) ? gen.q[t] : 0.0;
      sg.shv[r] = t <= d - 2 ? shift_at<T>(gen, k * (d - 1) + t) : T(0);
    }
  }

  __device__ __forceinline__ void stage_async(Staged<T> &sg, const typename TgtT<T>::type *tgt, int r,
                                              int64_t lbase, int nval) const {
    static_assert(sizeof(typename TgtT<T>::type) == 16 && sizeof(T) == 4, "FP32 staging");
    if (r < nval) {
      const int64_t t = d - 1 - (lbase + r);
      const bool has_u = t <= d - 2;
      const int64_t si = k * (d - 1) + t;
      cp_async_or_zero<16>(&sg.tg[r], &tgt[t], true);
      const bool vq = has_u && gen.q, vs = has_u && gen.shift32;
      cp_async_or_zero<8>(&sg.qv[r], vq ? (const void *)(gen.q + t) : (const void *)tgt, vq);
      cp_async_or_zero<4>(&sg.shv[r], vs ? (const void *)(gen.shift32 + si) : (const void *)tgt, vs);
    }
  }

  // tent-transformed point w_t of y-index t (as StepFp*::quantile forms it);
  // Sobol: from the staged integer xs (already XORed with the shift) when
  // `staged`, else generated here
  __device__ __forceinline__ double point_w(const Staged<T> &sg, int li, int64_t t, uint32_t xs,
                                            bool staged) const {
    double u;
    if (GEN == 0) {
      double x = __dmul_rn(jd, sg.qv[li]);
      x = x - floor(x);
      if (sizeof(T) == 4) {
        float uf = (float)sg.shv[li] + (float)x;
        uf = uf > 1.0f ? uf - 1.0f : uf;
        return (double)fabsf(fmaf(uf, 2.0f, -1.0f));
      }
      u = (double)sg.shv[li] + x;
      u = u > 1.0 ? u - 1.0 : u;
    } else {
      const int L = gen.n_bits;
      const uint64_t mask = (L >= 64) ? ~0ull : ((1ull << L) - 1);
      const uint64_t xi =
          (uint64_t)(staged ? xs : dbgz::sobol_warp(gen.V + t * 32, (uint64_t)(gen.sobol_first + gen.gen_base + j))) &
          mask;
      const uint64_t sh = staged ? 0ull : gen.ushift[k * (d - 1) + t] & mask;
      u = (double)((xi ^ sh) & mask) * ldexp(1.0, -L);
    }
    return fabs(fma(u, 2.0, -1.0));
  }

  // point_w in FP32 for the FP32 paths: the same floats as
  // StepFp32::quantile forms them (Richtmyer: the FP64 fraction, then FP32),
  // without a conversion back and forth through FP64
  __device__ __forceinline__ float point_w32(const Staged<T> &sg, int li, int64_t t, uint32_t xs,
                                             bool staged) const {
    if (GEN == 0) {
      double x = __dmul_rn(jd, sg.qv[li]);
      x = x - floor(x);
      float uf = (float)sg.shv[li] + (float)x;
      uf = uf > 1.0f ? uf - 1.0f : uf;
      return fabsf(fmaf(uf, 2.0f, -1.0f));
    }
    return (float)point_w(sg, li, t, xs, staged);
  }

  // adjoint of variable t given ybar_t; returns sbar_t (unit seed), records
  // the per-variable gradient terms (unit seed; accumulate scales by p).
  // The bound arguments and the normal densities are formed in T (FP32
  // paths: FP32 exp, as their y, s, dc are FP32 already); the reciprocals of
  // dc and of the density of y, which reach 1e30 and beyond for narrow
  // intervals, and everything multiplied by them stay FP64.
  __device__ __forceinline__ double variable(const typename TgtT<T>::type &tg, double w, bool has_u, T y, T s,
                                             T dc, bool clamp9, double &ga, double &gb, double &gu) const {
    const T r2 = T(1.4142135623730951), rpi = T(0.3989422804014327);
    const T inv_u = (T)tg.inv_u;  // 1 / (U_tt sqrt 2)
    const T xa = ((T)tg.a - s) * inv_u, xb = ((T)tg.b - s) * inv_u;
    const bool pa = !clamp9 || fabs(xa) < T(9), pb = !clamp9 || fabs(xb) < T(9);
    const T fa = pa ? rpi * exp(-xa * xa) : T(0);
    const T fb = pb ? rpi * exp(-xb * xb) : T(0);
    // d log(dc) / d dc; a dc of zero (weight zero) contributes nothing.  In
    // the FP32 paths the reciprocals are FP32 (2 ulp) while their results
    // stay in FP32 range, and FP64 divisions otherwise.
    double pex = 0.0, ubar = 0.0;
    if (sizeof(T) == 4) {
      if (dc > T(1e-30)) pex = (double)__fdividef(1.0f, (float)dc);
      else if (dc > T(0)) pex = 1.0 / (double)dc;
      if (has_u && fabs(y) < T(8.12585)) ubar = (double)ybar * (double)__fdividef(1.0f, (float)(rpi * exp(T(-0.5) * y * y)));
    } else {
      pex = dc > T(0) ? 1.0 / (double)dc : 0.0;
      if (has_u && fabs(y) < T(8.12585)) ubar = (double)ybar / (double)(rpi * exp(T(-0.5) * y * y));
    }
    const double eb = pex + ubar * w, cb = -pex + ubar * (1.0 - w);
    const double rU = (double)inv_u * 1.4142135623730951;  // 1 / U_tt
    ga = (fa != T(0)) ? cb * (double)fa * rU : 0.0;
    gb = (fb != T(0)) ? eb * (double)fb * rU : 0.0;
    const double al = (double)xa * 1.4142135623730951, be = (double)xb * 1.4142135623730951;
    gu = -((ga != 0.0 ? ga * al : 0.0) + (gb != 0.0 ? gb * be : 0.0));
    return -(ga + gb);
  }

  // FP32 form of variable() for the FP32 paths: every quantity in FP32.  A
  // result that leaves FP32 range (dc below 1e-36, or sensitivities beyond
  // 1e38) is not finite, and emit_from then redoes the warp in FP64.
  __device__ __forceinline__ float variable32(const typename TgtT<T>::type &tg, float w, bool has_u, float y,
                                              float s, float dc, bool clamp9, float &ga, float &gb,
                                              float &gu) const {
    // every quantity is formed unconditionally and chosen by selects: the
    // per-variable code stays free of branches
    const float r2 = 1.41421356237f, rpi = 0.398942280401f;
    const float inv_u = (float)tg.inv_u;
    const float xa = ((float)tg.a - s) * inv_u, xb = ((float)tg.b - s) * inv_u;
    // normal densities by the SFU's 2^z (0 at an infinite bound)
    const float ea = rpi * dbgz::exp2_sfu((xa * xa) * -1.44269504089f);
    const float eb_ = rpi * dbgz::exp2_sfu((xb * xb) * -1.44269504089f);
    const float fa = (!clamp9 || fabsf(xa) < 9.0f) ? ea : 0.0f;
    const float fb = (!clamp9 || fabsf(xb) < 9.0f) ? eb_ : 0.0f;
    const float rdc = __fdividef(1.0f, dc);
    const float pex = dc > 1e-36f ? rdc : (dc > 0.0f ? INFINITY : 0.0f);
    // ybar / phi(y) = ybar sqrt(2 pi) exp(y^2 / 2) (used for |y| < 8.13: below 2^48)
    const float ub = (float)ybar * 2.50662827463f * dbgz::exp2_sfu((y * y) * 0.72134752045f);
    const float ubar = (has_u && fabsf(y) < 8.12585f) ? ub : 0.0f;
    const float eb = fmaf(ubar, w, pex), cb = fmaf(ubar, 1.0f - w, -pex);
    const float rU = inv_u * r2;
    ga = fa != 0.0f ? cb * fa * rU : 0.0f;
    gb = fb != 0.0f ? eb * fb * rU : 0.0f;
    const float ta = ga != 0.0f ? ga * (xa * r2) : 0.0f, tb = gb != 0.0f ? gb * (xb * r2) : 0.0f;
    gu = -(ta + tb);
    return -(ga + gb);
  }

  // FP32 warp sums of the weighted terms (weights relative to the warp's
  // largest, scaled back in FP64)
  __device__ __forceinline__ void accumulate32(int64_t t, float ga, float gb, float gu) const {
    float f0 = wrel * ga, f1 = wrel * gb, f2 = wrel * gu;
    for (int o = 16; o > 0; o >>= 1) {
      f0 += __shfl_down_sync(0xffffffffu, f0, o);
      f1 += __shfl_down_sync(0xffffffffu, f1, o);
      f2 += __shfl_down_sync(0xffffffffu, f2, o);
    }
    if (lane == 0) {
      const int64_t row = ((tile - io.tile0) * 4 + warp) * d + t;
      io.ga[row] = (double)f0 * wmax;
      io.gb[row] = (double)f1 * wmax;
      io.gu[row] = (double)f2 * wmax;
    }
  }

  __device__ __forceinline__ void accumulate(int64_t t, double ga, double gb, double gu) const {
    if (sizeof(T) == 4) {
      float f0 = (float)(wrel * ga), f1 = (float)(wrel * gb), f2 = (float)(wrel * gu);
      const bool finite = isfinite(f0) && isfinite(f1) && isfinite(f2);
      if (__all_sync(0xffffffffu, finite)) {
        for (int o = 16; o > 0; o >>= 1) {
          f0 += __shfl_down_sync(0xffffffffu, f0, o);
          f1 += __shfl_down_sync(0xffffffffu, f1, o);
          f2 += __shfl_down_sync(0xffffffffu, f2, o);
        }
        if (lane == 0) {
          const int64_t row = ((tile - io.tile0) * 4 + warp) * d + t;
          io.ga[row] = (double)f0 * wmax;
          io.gb[row] = (double)f1 * wmax;
          io.gu[row] = (double)f2 * wmax;
        }
        return;
      }
      // a term beyond FP32 range somewhere in the warp: FP64 sums
    }
    double v0 = p * ga, v1 = p * gb, v2 = p * gu;
    for (int o = 16; o > 0; o >>= 1) {
      v0 += __shfl_down_sync(0xffffffffu, v0, o);
      v1 += __shfl_down_sync(0xffffffffu, v1, o);
      v2 += __shfl_down_sync(0xffffffffu, v2, o);
    }
    if (lane == 0) {
      const int64_t row = ((tile - io.tile0) * 4 + warp) * d + t;
      io.ga[row] = v0;
      io.gb[row] = v1;
      io.gu[row] = v2;
    }
  }

  // the factor-gradient GEMM's operand p * sbar_t (dense path); in FP32
  // rounded to the nearest TF32 value: the TF32 tensor cores drop the low 13
  // mantissa bits, which biases the products towards zero.  (The stored y's,
  // the other operand, are still truncated by the tensor cores; rounding them
  // too -- a write-back after the step has used y -- took the FP32
  // dP/dSigma error vs FP64 from 8.3e-4 to 6.5e-4 at d = 1000 for 2.2 ms, and
  // is not done.)
  __device__ __forceinline__ void store_gemm(int64_t t, bool, T, double psb) const {
    if (!io.sbar) return;
    __stcs(io.sbar + ga0 + t * io.stride(), sizeof(T) == 4 ? (T)tf32_rn((float)psb) : (T)psb);
  }
  __device__ __forceinline__ T emit_from(const Staged<T> &sg, int li, int64_t l, T y, T s, T dc, uint32_t xs) {
    const int64_t t = d - 1 - l;
    const bool has_u = t <= d - 2;
    const double w = has_u ? point_w(sg, li, t, xs, gen.sobol_staged != 0) : 0.0;
    if (sizeof(T) == 4) {
      float fa, fb, fu;
      const float sb = variable32(sg.tg[li], (float)w, has_u, (float)y, (float)s, (float)dc, true, fa, fb, fu);
      const bool fin = isfinite(sb) && isfinite(wrel * fa) && isfinite(wrel * fb) && isfinite(wrel * fu);
      if (__all_sync(0xffffffffu, fin)) {
        accumulate32(t, fa, fb, fu);
        store_gemm(t, has_u, y, p * (double)sb);
        return (T)sb;
      }
    }
    double ga, gb, gu;
    const double sb = variable(sg.tg[li], w, has_u, y, s, dc, true, ga, gb, gu);
    accumulate(t, ga, gb, gu);
    store_gemm(t, has_u, y, p * sb);
    return (T)sb;
  }
  __device__ __forceinline__ T emit(const Staged<T> &sg, int li, int64_t l, uint32_t xs = 0u) {
    const int64_t t = d - 1 - l;
    const T y = t <= d - 2 ? io.y[ga0 + t * io.stride()] : T(0);
    return emit_from(sg, li, l, y, io.s[ga0 + t * io.stride()], io.dc[ga0 + t * io.stride()], xs);
  }
  // chunked form: the stored state of the chunk's 8 steps (steps l0 .. l0+7,
  // n of them valid) is loaded before the first, so the loads overlap; in
  // the FP32 paths the weighted per-variable terms of the 8 steps are kept
  // and summed over the warp together in chunk_end
  T pre_y[8], pre_s[8], pre_dc[8];
  float acc_a[8], acc_b[8], acc_u[8];
  uint32_t fp64_done;  // steps of the chunk whose sums were written by the FP64 fallback (warp-uniform)
  __device__ __forceinline__ void chunk_begin(int64_t l0, int n) {
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      const int64_t t = d - 1 - (l0 + kk);
      const bool v = kk < n;
      pre_y[kk] = (v && t <= d - 2) ? __ldcs(io.y + ga0 + t * io.stride()) : T(0);
      pre_s[kk] = v ? __ldcs(io.s + ga0 + t * io.stride()) : T(0);
      pre_dc[kk] = v ? __ldcs(io.dc + ga0 + t * io.stride()) : T(0);
      acc_a[kk] = acc_b[kk] = acc_u[kk] = 0.0f;
    }
    fp64_done = 0u;
    // the next chunk's rows towards L2 while this chunk runs (the loads of the
    // next chunk_begin then wait on L2, not HBM: gradient 77.6 -> 75.7 ms at
    // d = 1000)
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      const int64_t t = d - 1 - (l0 + 8 + kk);
      if (t >= 1) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(io.y + ga0 + t * io.stride()));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(io.s + ga0 + t * io.stride()));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(io.dc + ga0 + t * io.stride()));
      }
    }
  }
  // emit_k without the per-step warp vote (FP32 paths): the FP32 terms in
  // any case, `bad` set where they are not finite; the loop then redoes the
  // chunk with emit_k from the chunk's saved state, which gives exactly what
  // emit_k alone would have given
  __device__ __forceinline__ T emit_k_fast(const Staged<T> &sg, int li, int64_t l, int kk, uint32_t xs) {
    const int64_t t = d - 1 - l;
    const bool has_u = t <= d - 2;
    const float w = has_u ? point_w32(sg, li, t, xs, gen.sobol_staged != 0) : 0.0f;
    float fa, fb, fu;
    const float sb = variable32(sg.tg[li], w, has_u, (float)pre_y[kk], (float)pre_s[kk], (float)pre_dc[kk], true, fa,
                                fb, fu);
    const float wa = wrel * fa, wb = wrel * fb, wu = wrel * fu;
    // one test for the four: an infinite or NaN term makes the sum so (a
    // finite sum that overflows only costs a redo)
    bad = bad || !isfinite((sb + wa) + (wb + wu));
    acc_a[kk] = wa;
    acc_b[kk] = wb;
    acc_u[kk] = wu;
    store_gemm(t, has_u, pre_y[kk], p * (double)sb);
    return (T)sb;
  }
  __device__ __forceinline__ T emit_k(const Staged<T> &sg, int li, int64_t l, int kk, uint32_t xs) {
    if (sizeof(T) != 4) return emit_from(sg, li, l, pre_y[kk], pre_s[kk], pre_dc[kk], xs);
    const int64_t t = d - 1 - l;
    const bool has_u = t <= d - 2;
    const double w = has_u ? point_w(sg, li, t, xs, gen.sobol_staged != 0) : 0.0;
    float fa, fb, fu;
    const float sb = variable32(sg.tg[li], (float)w, has_u, (float)pre_y[kk], (float)pre_s[kk],
                                (float)pre_dc[kk], true, fa, fb, fu);
    const float wa = wrel * fa, wb = wrel * fb, wu = wrel * fu;
    const bool fin = isfinite(sb) && isfinite(wa) && isfinite(wb) && isfinite(wu);
    if (__all_sync(0xffffffffu, fin)) {
      acc_a[kk] = wa;
      acc_b[kk] = wb;
      acc_u[kk] = wu;
      store_gemm(t, has_u, pre_y[kk], p * (double)sb);
      return (T)sb;
    }
    // a term beyond FP32 range in the warp: this step in FP64, its sums
    // written at once
    fp64_done |= 1u << kk;
    double ga, gb, gu;
    const double sbd = variable(sg.tg[li], w, has_u, pre_y[kk], pre_s[kk], pre_dc[kk], true, ga, gb, gu);
    accumulate(t, ga, gb, gu);
    store_gemm(t, has_u, pre_y[kk], p * sbd);
    return (T)sbd;
  }
  // sum of 8 values per lane over the 32 lanes of the warp, 8 sums at once:
  // three exchange-and-add rounds halve the values a lane holds (lanes
  // 16 apart split the 8 variables 4/4, then 8 apart 2/2, then 4 apart
  // 1/1), two plain rounds finish the sum; lane L ends with the sum of
  // variable (L >> 2) & 7.  9 shuffles instead of 40.
  static __device__ __forceinline__ float warp_sum8(float (&v)[8], int lane) {
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float send = b4 ? v[i] : v[i + 4], keep = b4 ? v[i + 4] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float send = b3 ? v[i] : v[i + 2], keep = b3 ? v[i + 2] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const float send = b2 ? v[0] : v[1], keep = b2 ? v[1] : v[0];
    float r = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    r += __shfl_xor_sync(0xffffffffu, r, 2);
    r += __shfl_xor_sync(0xffffffffu, r, 1);
    return r;
  }
  __device__ __forceinline__ void chunk_end(int64_t l0, int n) {
    if (sizeof(T) != 4 || n <= 0) return;
    const float sa = warp_sum8(acc_a, lane), sbv = warp_sum8(acc_b, lane), su = warp_sum8(acc_u, lane);
    const int kk = (lane >> 2) & 7;
    if ((lane & 3) == 0 && kk < n && !((fp64_done >> kk) & 1u)) {
      const int64_t t = d - 1 - (l0 + kk);
      const int64_t row = ((tile - io.tile0) * 4 + warp) * d + t;
      io.ga[row] = (double)sa * wmax;
      io.gb[row] = (double)sbv * wmax;
      io.gu[row] = (double)su * wmax;
    }
  }
  __device__ __forceinline__ void consume(const Staged<T> &, T r_sum, int, int64_t) { ybar = r_sum; }
  // the recursion's state between two steps (segments of the banded gradient)
  __device__ __forceinline__ void pack(double (&v)[4]) const {
    v[0] = (double)ybar;
    v[1] = v[2] = v[3] = 0.0;
  }
  __device__ __forceinline__ void unpack(const double (&v)[4]) { ybar = (T)v[0]; }

  __device__ __forceinline__ double tile_value(bool) { return 0.0; }
  // variable 0 after the last step: its CDF has no conditioning sum and no
  // clamp (src/qmc.jl:800-809); its point is QMC dimension 0
  __device__ __forceinline__ void tile_end(const typename TgtT<T>::type *tgt, int r, int, int64_t, bool) {
    Staged<T> sg0;
    sg0.qv[0] = gen.q ? gen.q[0] : 0.0;
    sg0.shv[0] = shift_at<T>(gen, k * (d - 1));
    const double w = point_w(sg0, 0, 0, 0u, false);
    const T y = io.y[ga0];
    double ga, gb, gu;
    variable(tgt[0], w, true, y, T(0), (T)io.dc1, false, ga, gb, gu);
    accumulate(0, ga, gb, gu);
  }
};

}  // namespace pol

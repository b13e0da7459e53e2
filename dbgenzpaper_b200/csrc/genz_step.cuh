// genz_step.cuh -- the per-sample, per-dimension step of the Genz
// sequential conditioning loop, shared by the SIMT and tensor-core loops.
//
// For one sample (point j of shift k) and one y-index l (QMC dimension l,
// conditioning variable l, target variable l+1) the reference does
// (src/qmc_generators.jl:137-204, src/qmc.jl:384-429):
//
//   u   = point(j, l) shifted (Richtmyer: + shift mod 1; Sobol: XOR shift)
//   w   = |2u - 1|                           (tent / baker transform)
//   u   = clamp(c + w dc, eps, 1 - eps)
//   y_l = sqrt(2) erfinv(2u - 1)             (= Phi^-1(u))
//   s   = sum_{i<=l} y_i U[i, l+1]           (the conditioning contraction)
//   c   = Phi((a_{l+1} - s)/U_{l+1,l+1}),  dc = Phi((b_{l+1} - s)/U) - c
//   p  *= dc
//
// Two numerics are provided:
//  * StepFp64: the reference's Float64 arithmetic (erf form or erfc form of
//    the CDF, the clamp to [-9, 9] in erf units, the same fma pattern).
//  * StepFp32: FP32 arithmetic kept close to the FP64 result where the
//    reference's Float32 loop loses digits (tail masses from normal32.cuh,
//    relative error < 3e-6 where they are above 1e-10; Phi^-1 of the smaller
//    tail from normal32.cuh, relative error < 4e-7): the state keeps both
//    tails -- lo = Phi(alpha), up = Phi(-beta)
//    -- and dc, so that u (when u <= 1/2) and 1 - u (otherwise) are formed
//    without cancellation and Phi^-1 is taken of the smaller one; dc is the
//    difference of two tails of the same side only when the interval lies
//    in one tail, and then in FP64 (erfc) if the FP32 difference would
//    cancel.  The weight product p stays FP64: FP32 would underflow where
//    the FP64 product is still normal (a product of d factors of about
//    1/2 leaves FP32's range at d ~ 150, FP64's at d ~ 1075); where P
//    itself is below FP64's range (e.g. 1000 bounds at marginal
//    probabilities 1e-3..1e-1) both give 0, as the reference does.
//    u is clamped to [eps64, 1 - eps64] like the Float64 reference.
#pragma once
#include "normal32.cuh"
#include <cuda_runtime.h>
#include <cstdint>
#include <cfloat>

namespace dbgz {

constexpr double kSqrt2 = 1.4142135623730951;

struct GenParams {
  int qmc_type;          // 0 Richtmyer, 1 Sobol
  int n_bits;
  int64_t gen_base;      // Richtmyer: n_base; Sobol: pass offset
  int64_t sobol_first;
  const double *q;       // Richtmyer generators (d-1)
  const double *shift64; // (d-1) x n_reps
  const float *shift32;  // (d-1) x n_reps
  const uint32_t *V;     // Sobol direction numbers (d-1) x 32
  const uint64_t *ushift;// (d-1) x n_reps
  const int64_t *gen_base_dev;  // when set, gen_base is read from here (device-driven passes)
  // Sobol, nonzero when the loop stages the integers of each block of
  // dimensions per tile (sobol_stage_block) and passes the point's integer,
  // already XORed with the shift's low 32 bits (n_bits <= 32: the shift
  // enters only there), into the step; zero: sobol_warp and the shift per
  // step.  Any first index: a tile's 128 points need the integers of 5
  // multiples of 32 and the terms of a 5-bit Gray code (SobolLane).
  int sobol_staged;
};

// Gray-code Sobol integer of point index idx in dimension l, computed by
// the 32 lanes of a warp together.  Precondition: every lane of the warp
// calls it at once for the same dimension, lane i with index idx0 + i (the
// loops give a warp 32 consecutive points).  Then
//   x(idx0) = XOR_k [bit k of gray(idx0)] V[k]   -- lane k supplies term k,
//   x(idx0 + i) = x(idx0) ^ XOR_{s=1..i} V[ctz(idx0 + s)]   -- Gray-code
// recurrence x(n) = x(n-1) ^ V[ctz(n)] as a prefix XOR over the lanes:
// two loads and ten shuffles per point instead of a loop over its set bits
// (same integers, exactly).
__device__ __forceinline__ uint32_t sobol_warp(const uint32_t *Vl, uint64_t idx) {
  const int lane = (int)(threadIdx.x & 31);
  const uint64_t i0 = idx - (uint64_t)lane;
  const uint32_t gw = (uint32_t)(i0 ^ (i0 >> 1));
  uint32_t x = ((gw >> lane) & 1u) ? __ldg(Vl + lane) : 0u;
  for (int o = 16; o > 0; o >>= 1) x ^= __shfl_xor_sync(0xffffffffu, x, o);
  const uint32_t lo = (uint32_t)idx;
  const int c = lo ? __ffs((int)lo) - 1 : 32;  // bits at 32 and above do not enter the 32-bit Gray code
  uint32_t t = (lane > 0 && c < 32) ? __ldg(Vl + c) : 0u;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, t, o);
    if (lane >= o) t ^= u;
  }
  return x ^ t;
}

// Staged Sobol integers of a 128-point tile with first index T (any T).
// Write T = B + o with B a multiple of 32 and o < 32; the point of tile row
// r < 128 has index B + 32 q + k with q = (o + r) >> 5 (0..4) and
// k = (o + r) & 31.  Since gray(N + k) = gray(N) ^ gray(k) for N a multiple
// of 32 and k < 32, and the integer is linear in the Gray code's bits, that
// integer is
//   x(B + 32 q) ^ x(gray(k) & 3) ^ x(gray(k) & 28).
// The five bases follow from x(B) by the recurrence over consecutive
// multiples of 32, x(32 (c + 1)) = x(32 c) ^ V[4] ^ V[5 + ctz(c + 1)]
// (of the 32 Gray-code steps between them, V[0..3] enter an even number of
// times, V[4] once, and the last step flips bit 5 + ctz(c + 1), which does
// not enter the 32-bit integer when it is 32 or more).  Per dimension li of a
// block, tab[li][0..16] holds: [q] = x(B + 32 q) ^ the tile's shift (low 32
// bits), [5 + a] = V[0], V[1] XORed by the bits of a, [9 + b] = V[2..4] by
// the bits of b.  A step then reads three words (SobolLane::at).
//
// sobol_stage_entries: the 32 lanes of one warp together fill entries
// li0 .. li0 + n - 1 of a block of 32: entry li < nv is dimension l0 + dir li
// when that lies in [0, lmax]; tile first index base0, shift row ush (the
// shift of dimension l at ush[l]).
constexpr int kSobolRow = 17;  // words per staged dimension
template <int UNROLL>
__device__ __forceinline__ void sobol_stage_entries(uint32_t (*tab)[kSobolRow], const uint32_t *V,
                                                    const uint64_t *ush, uint64_t base0, int64_t l0, int dir,
                                                    int64_t lmax, int nv, int li0, int n) {
  const uint64_t B = base0 & ~31ull;
  const uint32_t gB = (uint32_t)(B ^ (B >> 1));
  const int ln = (int)(threadIdx.x & 31);
  // lanes 1..4: bit 5 + ctz(c + ln) of the recurrence (c = B / 32)
  const int zb = (ln >= 1 && ln <= 4) ? 5 + __ffsll((long long)((B >> 5) + (uint64_t)ln)) - 1 : 32;
#pragma unroll UNROLL
  for (int q = 0; q < n; ++q) {
    const int li = li0 + q;
    const int64_t l = l0 + dir * li;
    const bool ok = li < nv && l >= 0 && l <= lmax;
    // x(B): lane k contributes V[k] when bit k of gray(B) is set
    const uint32_t vk = ok ? __ldg(V + l * 32 + ln) : 0u;
    uint32_t t = ((gB >> ln) & 1u) ? vk : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t ^= __shfl_xor_sync(0xffffffffu, t, o);
    uint32_t v[5];
#pragma unroll
    for (int e = 0; e < 5; ++e) v[e] = __shfl_sync(0xffffffffu, vk, e);
    // x(B + 32 ln) = x(B) ^ XOR_{s = 1..ln} (V[4] ^ V[5 + ctz(c + s)]), lanes 0..4
    const uint32_t vz = __shfl_sync(0xffffffffu, vk, zb & 31);
    uint32_t term = (ln >= 1 && ln <= 4) ? v[4] ^ (zb < 32 ? vz : 0u) : 0u;
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, term, o);
      if (ln >= o) term ^= u;
    }
    const uint32_t sh = (ln < 5 && ok) ? (uint32_t)__ldg(ush + l) : 0u;
    uint32_t x;
    if (ln < 5) {
      x = t ^ term ^ sh;
    } else if (ln < 9) {
      const int a = ln - 5;
      x = ((a & 1) ? v[0] : 0u) ^ ((a & 2) ? v[1] : 0u);
    } else {
      const int b = ln - 9;
      x = ((b & 1) ? v[2] : 0u) ^ ((b & 2) ? v[3] : 0u) ^ ((b & 4) ? v[4] : 0u);
    }
    if (ln < 17) tab[li][ln] = x;
  }
}
// The 128 threads r of a tile together (all lanes of their four warps), warp
// w filling entries 8w..8w+7.
__device__ __forceinline__ void sobol_stage_block(uint32_t (*tab)[kSobolRow], const uint32_t *V,
                                                  const uint64_t *ush, uint64_t base0, int64_t l0, int dir,
                                                  int64_t lmax, int nv, int r) {
  sobol_stage_entries<8>(tab, V, ush, base0, l0, dir, lmax, nv, 8 * (r >> 5), 8);
}

// The shifted integer of tile row r in block dimension li, for the tile
// whose first point index is base0 (sobol_stage_block).
struct SobolLane {
  uint32_t q, a, b;  // base slot, gray(k) & 3, gray(k) >> 2
  __device__ __forceinline__ SobolLane(int r, uint64_t base0) {
    const uint32_t s = (uint32_t)(base0 & 31u) + (uint32_t)r;  // o + r < 160
    const uint32_t k = s & 31u;
    const uint32_t g = k ^ (k >> 1);
    q = s >> 5;
    a = g & 3u;
    b = g >> 2;
  }
  __device__ __forceinline__ uint32_t at(const uint32_t (*tab)[kSobolRow], int li) const {
    const uint32_t *t = tab[li];
    return t[q] ^ t[5 + a] ^ t[9 + b];
  }
};

// w = |2u - 1| and w1 = 2 min(u, 1 - u) of the Sobol point u = X 2^-L
// (X < 2^L, 1 <= L <= 32), rounded to FP32.  Both are exact multiples of
// 2^-(L-1) with integer parts |X - 2^(L-1)| and min(X, 2^L - X) <= 2^31, so
// forming them on the integer and rounding once gives the same floats as
// forming u in FP64 first (checked for every L on random and edge X).
__device__ __forceinline__ void sobol_tent_f32(uint32_t X, int L, float &w, float &w1) {
  const uint32_t half = 1u << (L - 1);
  const uint32_t dd = X >= half ? X - half : half - X;
  const uint32_t mm = X <= half ? X : (uint32_t)((1ull << L) - X);
  const float sc = __int_as_float((127 - (L - 1)) << 23);  // 2^-(L-1)
  w = __uint2float_rn(dd) * sc;
  w1 = __uint2float_rn(mm) * sc;
}

// The same integer by one thread alone (loop over the set bits).
__device__ __forceinline__ uint32_t sobol_int(const uint32_t *Vl, uint64_t idx) {
  uint32_t g = (uint32_t)(idx ^ (idx >> 1));
  uint32_t x = 0;
  while (g) {
    int k = __ffs(g) - 1;
    x ^= __ldg(Vl + k);
    g &= g - 1;
  }
  return x;
}

// ---------------------------------------------------------------- FP64 ---
struct StepFp64 {
  double c, dc;
  double p;
  __device__ __forceinline__ void init(double c1, double dc1, double /*up1*/) {
    c = c1;
    dc = dc1;
    p = dc1;
  }
  // Returns y_l for QMC dimension l of sample (point index j in the pass,
  // 0-based; shift k).
  template <bool kIntTent = true>  // (no effect in FP64)
  __device__ __forceinline__ double quantile(const GenParams &g, int64_t d, int64_t j, int64_t k,
                                             int64_t l, double qv, double shiftv, uint32_t x0) const {
    double u;
    if (g.qmc_type == 0) {
      double x = __dmul_rn((double)(g.gen_base + j + 1), qv);
      x = x - floor(x);
      u = shiftv + x;
      u = u > 1.0 ? u - 1.0 : u;
    } else {
      const int L = g.n_bits;
      const uint64_t mask = (L >= 64) ? ~0ull : ((1ull << L) - 1);
      const uint32_t xw = g.sobol_staged ? x0 : sobol_warp(g.V + l * 32, (uint64_t)(g.sobol_first + g.gen_base + j));
      uint64_t xi = (uint64_t)xw & mask;
      uint64_t sh = g.sobol_staged ? 0ull : g.ushift[k * (d - 1) + l] & mask;
      u = (double)((xi ^ sh) & mask) * ldexp(1.0, -L);
    }
    u = fabs(fma(u, 2.0, -1.0));
    u = fma(u, dc, c);
    u = fmin(fmax(u, DBL_EPSILON), 1.0 - DBL_EPSILON);
    double v = fma(2.0, u, -1.0);
    return kSqrt2 * erfinv(v);
  }
  __device__ __forceinline__ void set_form(int) {}
  // the state between two steps, as four doubles (checkpoints)
  __device__ __forceinline__ void pack(double (&v)[4]) const {
    v[0] = c;
    v[1] = dc;
    v[2] = p;
    v[3] = 0.0;
  }
  __device__ __forceinline__ void unpack(const double (&v)[4]) {
    c = v[0];
    dc = v[1];
    p = v[2];
  }
  __device__ __forceinline__ void cdf(double s, double a, double b, double inv_u, int erfc_form) {
    double cv = (a - s) * inv_u;
    double dv = (b - s) * inv_u;
    cv = fmax(fmin(cv, 9.0), -9.0);
    dv = fmax(fmin(dv, 9.0), -9.0);
    if (!erfc_form) {
      cv = 0.5 * (1.0 + erf(cv));
      dv = 0.5 * (1.0 + erf(dv)) - cv;
    } else {
      double c_val = 0.5 * erfc(-cv);
      dv = 0.5 * erfc(-dv) - c_val;
      cv = c_val;
    }
    c = cv;
    dc = dv;
    p *= dv;
  }
};

// The FP64 step of a problem whose lower bounds are all -inf (P(X <= b)):
// the lower argument is always clamped to -9, so its CDF value is one
// constant, evaluated once per sample by the same function from the same
// argument (hidden from constant folding) -- the same bits as the general
// step, one erf (or erfc) per step fewer.
struct StepFp64LowerInf : StepFp64 {
  double cinf;  // the lower bound's CDF value in the pass's form (set_form)
  __device__ __forceinline__ void set_form(int erfc_form) {
    double m9 = -9.0;
    asm volatile("" : "+d"(m9));
    cinf = erfc_form ? 0.5 * erfc(-m9) : 0.5 * (1.0 + erf(m9));
  }
  __device__ __forceinline__ void cdf(double s, double /*a*/, double b, double inv_u, int erfc_form) {
    double dv = (b - s) * inv_u;
    dv = fmax(fmin(dv, 9.0), -9.0);
    double cv;
    if (!erfc_form) {
      cv = cinf;
      dv = 0.5 * (1.0 + erf(dv)) - cv;
    } else {
      const double c_val = cinf;
      dv = 0.5 * erfc(-dv) - c_val;
      cv = c_val;
    }
    c = cv;
    dc = dv;
    p *= dv;
  }
};

// ---------------------------------------------------------------- FP32 ---
// Phi(-x0) - Phi(-x1) = (erfc(x0) - erfc(x1)) / 2 for 0 <= x0 <= x1 (erf
// units) in FP64: the FP32 difference of two close tail masses cancels.
// Rarely taken; kept out of line so the unrolled loop stays small.
static __device__ __noinline__ float same_tail_mass64(float x0, float x1) {
  return (float)(0.5 * (erfc((double)x0) - erfc((double)x1)));
}

struct StepFp32 {
  float lo, up, dc;  // Phi(alpha), Phi(-beta), Phi(beta) - Phi(alpha)
  double p;
  __device__ __forceinline__ void init(double c1, double dc1, double up1) {
    lo = (float)c1;
    dc = (float)dc1;
    up = (float)up1;
    p = dc1;
  }
  // kIntTent: the Sobol tent transform on the integer (sobol_tent_f32), else
  // through an FP64 u -- the same floats; the pass that stores its state for
  // the adjoint keeps the FP64 form (measured on the banded d = 10^4,
  // bandwidth 64 workload at 2^14 x 10 Sobol points: its
  // gradient call 125.1 ms against 146.4 ms with the integer form)
  template <bool kIntTent = true>
  __device__ __forceinline__ float quantile(const GenParams &g, int64_t d, int64_t j, int64_t k,
                                            int64_t l, double qv, float shiftv, uint32_t x0) const {
    float w, w1;
    if (g.qmc_type == 0) {
      double x = __dmul_rn((double)(g.gen_base + j + 1), qv);
      x = x - floor(x);
      float u = shiftv + (float)x;
      u = u > 1.0f ? u - 1.0f : u;
      w = fabsf(fmaf(u, 2.0f, -1.0f));
      w1 = 2.0f * fminf(u, 1.0f - u);  // 1 - |2u - 1|
    } else if (kIntTent) {
      // n_bits <= 32: the shifted integer has at most 32 bits
      const int L = g.n_bits;
      const uint32_t mask = L >= 32 ? 0xffffffffu : ((1u << L) - 1u);
      const uint32_t xw = g.sobol_staged ? x0 : sobol_warp(g.V + l * 32, (uint64_t)(g.sobol_first + g.gen_base + j));
      const uint32_t sh = g.sobol_staged ? 0u : (uint32_t)g.ushift[k * (d - 1) + l];
      sobol_tent_f32((xw ^ sh) & mask, L, w, w1);
    } else {
      const int L = g.n_bits;
      const uint64_t mask = (L >= 64) ? ~0ull : ((1ull << L) - 1);
      const uint32_t xw = g.sobol_staged ? x0 : sobol_warp(g.V + l * 32, (uint64_t)(g.sobol_first + g.gen_base + j));
      const uint64_t xi = (uint64_t)xw & mask;
      const uint64_t sh = g.sobol_staged ? 0ull : g.ushift[k * (d - 1) + l] & mask;
      const double u = (double)((xi ^ sh) & mask) * ldexp(1.0, -L);
      w = (float)fabs(fma(u, 2.0, -1.0));
      w1 = (float)(2.0 * fmin(u, 1.0 - u));
    }
    const float kEps = (float)DBL_EPSILON;
    // u = lo + w dc when that is <= 1/2, else 1 - u = up + (1 - w) dc;
    // Phi^-1 is taken of the smaller one (one call site keeps the code small)
    const float t = fmaf(w, dc, lo);
    const bool lower = t <= 0.5f;
    const float arg = lower ? t : fmaf(w1, dc, up);
    const float y = phi_inv_lower_f32(fmaxf(arg, kEps));
    return lower ? y : -y;
  }
  __device__ __forceinline__ void set_form(int) {}
  // the state between two steps, as four doubles (checkpoints; the floats
  // are exact in double)
  __device__ __forceinline__ void pack(double (&v)[4]) const {
    v[0] = lo;
    v[1] = up;
    v[2] = dc;
    v[3] = p;
  }
  __device__ __forceinline__ void unpack(const double (&v)[4]) {
    lo = (float)v[0];
    up = (float)v[1];
    dc = (float)v[2];
    p = v[3];
  }
  // The tails and the FP32 difference of the interval's masses; need64: the
  // interval lies in one tail and that difference cancels (the masses are
  // within a factor 2).
  __device__ __forceinline__ float cdf_core(float s, float a, float b, float inv_u, float &x0, float &x1,
                                            bool &need64) {
    const float xa = fminf(fmaxf((a - s) * inv_u, -9.0f), 9.0f);
    const float xb = fminf(fmaxf((b - s) * inv_u, -9.0f), 9.0f);
    const float ea = tail_mass_f32(fabsf(xa));  // mass beyond |alpha| on its side
    const float eb = tail_mass_f32(fabsf(xb));
    // both bounds in the upper tail (hi_t), both in the lower tail (lo_t), or
    // alpha < 0 < beta; selects rather than branches (the step is a serial
    // chain per sample, and branch resolution stalls it)
    const bool hi_t = xa >= 0.0f, lo_t = !hi_t && xb <= 0.0f;
    const float d = hi_t ? ea - eb : (lo_t ? eb - ea : (1.0f - ea) - eb);
    need64 = (hi_t && eb > 0.5f * ea) || (lo_t && ea > 0.5f * eb);
    x0 = hi_t ? xa : -xb;
    x1 = hi_t ? xb : -xa;
    lo = hi_t ? 1.0f - ea : ea;
    up = lo_t ? 1.0f - eb : eb;
    return d;
  }
  // The exact factor of a step whose FP32 difference cancels, from the same
  // inputs (the same x0, x1 bits as cdf_core).
  static __device__ __forceinline__ float tail_exact(float s, float a, float b, float inv_u) {
    const float xa = fminf(fmaxf((a - s) * inv_u, -9.0f), 9.0f);
    const float xb = fminf(fmaxf((b - s) * inv_u, -9.0f), 9.0f);
    const bool hi_t = xa >= 0.0f;
    return same_tail_mass64(hi_t ? xa : -xb, hi_t ? xb : -xa);
  }
  __device__ __forceinline__ void cdf(float s, float a, float b, float inv_u, int /*erfc_form*/) {
    float x0, x1;
    bool need64;
    float d = cdf_core(s, a, b, inv_u, x0, x1, need64);
    if (need64) d = same_tail_mass64(x0, x1);
    dc = d;
    p *= (double)d;
  }
  // cdf without the branch: where the FP32 difference cancels, dc keeps it
  // and the weight is not multiplied; the caller multiplies the exact factor
  // (tail_exact) in later.  The next step's u takes dc at the FP32 tail
  // masses' own accuracy either way (in one tail, u or 1 - u lies between
  // the two masses and dc's absolute error is at most theirs); the weight
  // needs dc to relative accuracy, so its factor waits for the exact value.
  // Returns whether the factor was left out.
  __device__ __forceinline__ bool cdf_deferred(float s, float a, float b, float inv_u) {
    float x0, x1;
    bool need64;
    const float d = cdf_core(s, a, b, inv_u, x0, x1, need64);
    dc = d;
    p *= (double)(need64 ? 1.0f : d);
    return need64;
  }
};

// The FP32 step of a problem whose lower bounds are all -inf: the lower tail
// argument is always -9, its tail mass one constant computed once per sample
// by the same function from the same argument -- the same bits as StepFp32,
// one tail mass per step fewer.
struct StepFp32LowerInf : StepFp32 {
  float ea9;
  __device__ __forceinline__ void init(double c1, double dc1, double up1) {
    StepFp32::init(c1, dc1, up1);
    float nine = 9.0f;
    asm volatile("" : "+f"(nine));
    ea9 = tail_mass_f32(nine);
  }
  __device__ __forceinline__ float cdf_core(float s, float b, float inv_u, bool &need64) {
    const float xb = fminf(fmaxf((b - s) * inv_u, -9.0f), 9.0f);
    const float ea = ea9;
    const float eb = tail_mass_f32(fabsf(xb));
    // alpha = -9 < 0: the interval is in the lower tail or straddles 0
    const bool lo_t = xb <= 0.0f;
    const float d = lo_t ? eb - ea : (1.0f - ea) - eb;
    need64 = lo_t && ea > 0.5f * eb;
    lo = ea;
    up = lo_t ? 1.0f - eb : eb;
    return d;
  }
  static __device__ __forceinline__ float tail_exact(float s, float /*a*/, float b, float inv_u) {
    const float xb = fminf(fmaxf((b - s) * inv_u, -9.0f), 9.0f);
    return same_tail_mass64(-xb, 9.0f);
  }
  __device__ __forceinline__ void cdf(float s, float /*a*/, float b, float inv_u, int /*erfc_form*/) {
    bool need64;
    float d = cdf_core(s, b, inv_u, need64);
    if (need64) d = tail_exact(s, 0.0f, b, inv_u);
    dc = d;
    p *= (double)d;
  }
  __device__ __forceinline__ bool cdf_deferred(float s, float /*a*/, float b, float inv_u) {
    bool need64;
    const float d = cdf_core(s, b, inv_u, need64);
    dc = d;
    p *= (double)(need64 ? 1.0f : d);
    return need64;
  }
};

// Step types of a working type, general and for all-lower-bounds -inf.
template <typename T, bool kLowerInf>
struct StepSel;
template <>
struct StepSel<double, false> {
  using type = StepFp64;
};
template <>
struct StepSel<double, true> {
  using type = StepFp64LowerInf;
};
template <>
struct StepSel<float, false> {
  using type = StepFp32;
};
template <>
struct StepSel<float, true> {
  using type = StepFp32LowerInf;
};

}  // namespace dbgz

// points.cu -- QMC point sets.
//
//  * Richtmyer lattice (reference src/qmc_generators.jl:300-325):
//    X[i,j] = frac((n0 + i) q_j), q_j = frac(sqrt(p_j)), p_j the j-th prime,
//    evaluated in FP64 (the product is a single rounded multiply; no FMA
//    contraction so the fraction is bit-identical to the reference).
//  * Sobol on the 32-bit grid (sobol_mat! + copyt_as_UInt64!,
//    src/qmc_generators.jl:331-352): Gray-code order (Antonov-Saleev),
//    x_n = XOR of v_k over the set bits k of n ^ (n >> 1).  Each point is
//    computed from its index directly, so any range of points is generated
//    without sequential state.
//
// The integration kernels do not read these matrices: they generate the
// point of (sample, dimension) in registers.  These kernels back the
// richtmyer_mat!/sobol_mat! entry points of the ABI.
#include "internal.cuh"
#include <algorithm>

namespace {

__global__ void k_richtmyer(int64_t m, int64_t n, const double *q, int64_t n0, double *X) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t j = blockIdx.y;
  if (i >= m) return;
  double x = __dmul_rn((double)(n0 + i + 1), q[j]);
  X[j * m + i] = x - floor(x);
}

__global__ void k_sobol(int64_t m, int64_t dims, const uint32_t *V, int64_t first, uint32_t *X) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t i = blockIdx.y;
  if (j >= m) return;
  uint64_t idx = (uint64_t)(first + j);
  uint32_t g = (uint32_t)(idx ^ (idx >> 1));
  const uint32_t *Vi = V + i * 32;
  uint32_t x = 0;
  while (g) {
    int k = __ffs(g) - 1;
    x ^= Vi[k];
    g &= g - 1;
  }
  X[i * m + j] = x;
}

// ---- host: primitive polynomials and direction numbers -------------------

uint64_t polymulmod(uint64_t a, uint64_t b, uint64_t p, int deg) {
  uint64_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    b >>= 1;
    a <<= 1;
    if (a >> deg & 1) a ^= p;
  }
  return r;
}
uint64_t polypowmod(uint64_t base, uint64_t e, uint64_t p, int deg) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = polymulmod(r, base, p, deg);
    base = polymulmod(base, base, p, deg);
    e >>= 1;
  }
  return r;
}
// p has degree deg (bit deg set, bit 0 set).  Primitive iff the order of x
// modulo p is exactly 2^deg - 1.
bool is_primitive(uint64_t p, int deg) {
  if (deg == 1) return p == 3;
  uint64_t order = (1ull << deg) - 1;
  uint64_t x = 2;
  if (polypowmod(x, order, p, deg) != 1) return false;
  uint64_t n = order;
  for (uint64_t f = 2; f * f <= n; ++f) {
    if (n % f) continue;
    while (n % f == 0) n /= f;
    if (polypowmod(x, order / f, p, deg) == 1) return false;
  }
  if (n > 1 && polypowmod(x, order / n, p, deg) == 1) return false;
  return true;
}

uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" int dbgz_sobol_dirnums(int64_t dims, uint32_t *V) {
  if (dims < 0 || (dims > 0 && !V)) return DBGZ_ERR_INVALID_ARGUMENT;
  if (dims > (1 << 20)) return DBGZ_ERR_DIMENSION;
  uint64_t seed = 0x5DB6E2F1C0FFEE01ull;
  int64_t made = 0;
  if (dims > 0) {  // van der Corput
    for (int k = 0; k < 32; ++k) V[k] = 1u << (31 - k);
    made = 1;
  }
  for (int deg = 1; made < dims && deg < 31; ++deg) {
    for (uint64_t p = (1ull << deg) | 1ull; p < (2ull << deg) && made < dims; p += 2) {
      if (!is_primitive(p, deg)) continue;
      uint32_t mk[33];
      mk[1] = 1;
      for (int k = 2; k <= deg && k <= 32; ++k) {
        uint32_t r = (uint32_t)(splitmix64(seed) % (1ull << (k - 1)));
        mk[k] = 2 * r + 1;  // odd, < 2^k
      }
      for (int k = deg + 1; k <= 32; ++k) {
        uint32_t v = mk[k - deg] ^ (mk[k - deg] << deg);
        for (int t = 1; t < deg; ++t)
          if ((p >> (deg - t)) & 1u) v ^= mk[k - t] << t;
        mk[k] = v;
      }
      uint32_t *Vi = V + made * 32;
      for (int k = 1; k <= 32; ++k) Vi[k - 1] = mk[k] << (32 - k);
      ++made;
    }
  }
  return made == dims ? DBGZ_OK : DBGZ_ERR_DIMENSION;
}

extern "C" int dbgz_sqrt_primes(int64_t n, double *q) {
  if (n < 0 || (n > 0 && !q)) return DBGZ_ERR_INVALID_ARGUMENT;
  int64_t p = 1;
  for (int64_t i = 0; i < n; ++i) {
    p = p + 1;  // nextprime(p + 1)
    for (;; ++p) {
      bool prime = p >= 2;
      for (int64_t f = 2; f * f <= p && prime; ++f)
        if (p % f == 0) prime = false;
      if (prime) break;
    }
    double sp = sqrt((double)p);
    q[i] = sp - floor(sp);
  }
  return DBGZ_OK;
}

int dbgz_richtmyer_dev(dbgz_ctx *ctx, int64_t m, int64_t n, const double *q, int64_t n0,
                       double *X) {
  if (m <= 0 || n <= 0) return DBGZ_OK;
  dim3 grid((unsigned)((m + 255) / 256), (unsigned)n);
  k_richtmyer<<<grid, 256, 0, ctx->stream>>>(m, n, q, n0, X);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_sobol_dev(dbgz_ctx *ctx, int64_t m, int64_t dims, const uint32_t *V, int64_t first,
                   uint32_t *X) {
  if (m <= 0 || dims <= 0) return DBGZ_OK;
  dim3 grid((unsigned)((m + 255) / 256), (unsigned)dims);
  k_sobol<<<grid, 256, 0, ctx->stream>>>(m, dims, V, first, X);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

// noalloc.cu -- one FP64 integration pass without any device allocation.
//
// Some callers cannot let a library allocate device memory: a host framework
// that owns every device buffer and hands them to the library (an XLA/JAX
// custom call, a Julia program whose GPU memory is CUDA.jl's pool), or a
// latency-critical caller for whom cudaMalloc/cudaFree would synchronise the
// whole device.  dbgz_pnorm_pass_noalloc serves them: the caller passes its
// inputs and outputs as device pointers, and the scratch the SIMT loop needs
// (per-target constants, the per-CTA y workspace, the per-tile partial sums)
// lives in one file-scope __device__ array of fixed size compiled into the
// library.  Every GPU that loads the library holds that array until exit.
//
// The kernels are the SIMT loop's own templates (loop_simt_kernels.cuh);
// only the source of the first dimension's (c, dc) differs: it is computed
// on the device into the array instead of on the host.
#include "loop_simt_kernels.cuh"
#include <cuda.h>
#include <algorithm>
#include <mutex>

using namespace simt;

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;       // 32 MiB in total
constexpr size_t kHdrBytes = 256;                         // c1, dc1
constexpr size_t kTgtBytes = size_t(768) << 10;           // per-target constants
constexpr size_t kPartBytes = size_t(1) << 20;            // per-tile partial sums
constexpr size_t kYOffset = kHdrBytes + kTgtBytes + kPartBytes;
constexpr size_t kYBytes = kScratchBytes - kYOffset;      // per-CTA y workspace
constexpr int64_t kMaxD = 8192;
constexpr int64_t kMaxTiles = int64_t(kPartBytes / sizeof(double));
static_assert(kMaxD * sizeof(TargetParams64) <= kTgtBytes, "target region too small");

// The scratch.  Host code must not use this name as an address: it is a
// host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// The array's device address belongs to a CUDA context (the module is loaded
// per context), so the cache is keyed on the current context's unique id
// (cuCtxGetId: a new context, also the primary context re-created after
// cudaDeviceReset, gets a new id), not on the device ordinal.
struct DeviceSlot {
  unsigned long long ctx_id = 0;
  bool used = false;
  unsigned char *ptr = nullptr;
  int per_sm = 0;
  int num_sms = 0;
};
constexpr int kSlots = 64;
std::mutex g_mu;
DeviceSlot g_slots[kSlots];
int g_next_slot = 0;

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// The unique id of the calling thread's current context (0 on failure).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = (CtxGetCurrentFn)p;
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)p;
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// The FP64 step whose first-dimension (c, dc) is read from the array header.
struct StepFp64Scratch : dbgz::StepFp64 {
  __device__ __forceinline__ void init(double, double, double) {
    const double *hdr = reinterpret_cast<const double *>(g_noalloc_scratch);
    dbgz::StepFp64::init(hdr[0], hdr[1], 0.0);
  }
};

using NoallocPolicy = pol::Forward<double, DBGZ_QMC_RICHTMYER, false, StepFp64Scratch>;

// Per-target constants and the first dimension's CDF values
// (src/qmc.jl:800-809, erf form).
__global__ void k_noalloc_setup(const double *U, int64_t d, const double *a, const double *b,
                                TargetParams64 *tgt, double *hdr) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const double c2 = sqrt(2.0);
  if (t < d) tgt[t] = TargetParams64{a[t], b[t], 1.0 / (U[t * d + t] * c2)};
  if (t == 0) {
    double arg_a = a[0] / (U[0] * c2), arg_b = b[0] / (U[0] * c2);
    hdr[0] = 0.5 * (1.0 + erf(arg_a));
    hdr[1] = 0.5 * (erf(arg_b) - erf(arg_a));
  }
}

int setup_device(int dev, DeviceSlot &slot) {
  // the context must be current (cudaGetDevice made the runtime's primary
  // context current if the caller had none)
  const unsigned long long id = current_context_id();
  if (!id) return DBGZ_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  for (int i = 0; i < kSlots; ++i)
    if (g_slots[i].used && g_slots[i].ctx_id == id) {
      slot = g_slots[i];
      return DBGZ_OK;
    }
  DeviceSlot s;
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return DBGZ_ERR_CUDA;
  }
  s.ptr = (unsigned char *)p;
  auto kern = k_genz_simt<double, NoallocPolicy>;
  const int smem = (int)sizeof(SimtSmem<double>);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s.per_sm, kern, NT, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&s.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      s.per_sm < 1) {
    cudaGetLastError();
    return DBGZ_ERR_CUDA;
  }
  s.ctx_id = id;
  s.used = true;
  g_slots[g_next_slot] = s;  // round robin over the slots once all are taken
  g_next_slot = (g_next_slot + 1) % kSlots;
  slot = s;
  return DBGZ_OK;
}

}  // namespace

extern "C" int dbgz_pnorm_pass_noalloc(int64_t d, const double *U, const double *a,
                                       const double *b, const double *q, const double *shifts,
                                       int64_t m, int64_t n_reps, int64_t n_base,
                                       double *qmc_reps, void *stream) {
  if (!U || !a || !b || !q || !shifts || !qmc_reps || m < 1 || n_reps < 1 || n_base < 0)
    return DBGZ_ERR_INVALID_ARGUMENT;
  if (d < 2 || d > kMaxD) return DBGZ_ERR_DIMENSION;
  // tiles per shift without overflow (m + TS - 1 could wrap), and the tile
  // count checked before it is formed (tps * n_reps could wrap)
  const int64_t tps = m / TS + (m % TS != 0);
  if (n_reps > kMaxTiles || tps > kMaxTiles / n_reps) return DBGZ_ERR_DIMENSION;
  const int64_t n_tiles = tps * n_reps;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return DBGZ_ERR_CUDA;
  }
  DeviceSlot slot;
  if (setup_device(dev, slot) != DBGZ_OK) return DBGZ_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;

  const int64_t Dp = ((d - 1 + G - 1) / G) * G;
  const size_t y_per_cta = sizeof(double) * (size_t)Dp * TS;
  int64_t grid = std::min<int64_t>(n_tiles, (int64_t)slot.per_sm * slot.num_sms);
  grid = std::min<int64_t>(grid, (int64_t)(kYBytes / y_per_cta));
  if (grid < 1) return DBGZ_ERR_DIMENSION;

  double *hdr = reinterpret_cast<double *>(slot.ptr);
  TargetParams64 *tgt = reinterpret_cast<TargetParams64 *>(slot.ptr + kHdrBytes);
  double *partials = reinterpret_cast<double *>(slot.ptr + kHdrBytes + kTgtBytes);
  double *yws = reinterpret_cast<double *>(slot.ptr + kYOffset);

  k_noalloc_setup<<<(unsigned)((d + 127) / 128), 128, 0, st>>>(U, d, a, b, tgt, hdr);
  SimtParams<double> P{};
  P.d = d;
  P.m = m;
  P.n_reps = n_reps;
  P.tiles_per_shift = tps;
  P.n_tiles = n_tiles;
  P.Dp = Dp;
  P.gen.qmc_type = DBGZ_QMC_RICHTMYER;
  P.gen.n_bits = 32;
  P.gen.gen_base = n_base;
  P.gen.q = q;
  P.gen.shift64 = shifts;
  P.U = U;
  P.tgt = tgt;
  P.cdf_form = DBGZ_CDF_ERF;
  P.yws = yws;
  P.partials = partials;
  k_genz_simt<double, NoallocPolicy><<<(unsigned)grid, NT, sizeof(SimtSmem<double>), st>>>(P);
  // the output accumulates a running mean with weight 0 for a first pass:
  // clear it so that stale or uninitialised contents cannot leak in
  if (cudaMemsetAsync(qmc_reps, 0, sizeof(double) * n_reps, st) != cudaSuccess) {
    cudaGetLastError();
    return DBGZ_ERR_CUDA;
  }
  k_finalize<<<(unsigned)((n_reps + 127) / 128), 128, 0, st>>>(partials, tps, n_reps, 0, m,
                                                                 qmc_reps);
  if (cudaGetLastError() != cudaSuccess) return DBGZ_ERR_CUDA;
  return DBGZ_OK;
}

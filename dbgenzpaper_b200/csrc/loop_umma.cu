// loop_umma.cu -- the dense Genz integration loop with the conditioning
// contraction on tcgen05 tensor cores (split-BF16 or TF32, FP32 accumulate
// in TMEM) and the sequential per-dimension step on CUDA cores.
//
// Replaces qmc_loop!(::QMCData) (reference src/qmc.jl:315-444) for
// T = Float32-class precision; the per-sample step is genz_step.cuh's
// StepFp32 (FP32 special functions, FP64 weight product, FP64 tails).
//
// Decomposition.  One CTA owns a tile of 128 samples (128 consecutive points
// of one shift) = the 128 TMEM lanes = the M of every MMA.  y-indices are
// processed in blocks of 32; TMEM holds the partial sums of the next targets
// as two halves of 128 columns (half h = the targets of blocks 4h..4h+3):
//   * block X: the 128 sample threads read their 32 partial sums of the
//     block's targets from TMEM (tcgen05.ld), run the 32 sequential steps
//     with in-register updates for the block's own triangle, and write their
//     y's (split hi/lo BF16, or TF32) as the A tile of the next MMA in shared
//     memory (the producer stores it to a per-CTA workspace in HBM/L2 when a
//     later half's re-initialisation reads it);
//   * after block X: S[:, targets of blocks X+1 .. end of the next half] +=
//     Y_X U[X rows, ...] on the tensor cores -- first the 32 columns the next
//     block needs (committed to their own barrier so the sample threads can
//     go on), then the rest, which overlaps with the next block's steps;
//     after the last block of a half also the first (overwriting)
//     contribution to the half after next, in the columns just freed;
//   * re-initialisation of half g >= 2: the contributions of y-blocks
//     0 .. 4g-6, a K = 32 GEMM chunk per y-block (A streamed back from the
//     workspace, B the U^T rows of half g, both by TMA), issued a quarter
//     per block during the blocks before half g is needed.
// Warp roles: warps 0-3 sample threads, warp 4 TMEM owner + MMA issuer,
// warp 5 TMA producer.  Every wait is bounded (sm100.cuh); a timeout sets
// DBGZ_ERR_TIMEOUT in the status word and the CTA drains and leaves.
#include <cuda.h>
#include <algorithm>
#include <type_traits>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "genz_step.cuh"
#include "sm100.cuh"
#include "policies.cuh"

namespace {

using namespace sm100;

constexpr int TS = 128;    // samples per tile = TMEM lanes = MMA M
constexpr int BK = 32;     // y-indices per block
constexpr int NT = 192;    // 4 sample warps + MMA warp + producer warp
constexpr int kMmaWarp = 4, kProdWarp = 5;
constexpr int kBarScalar = 1;  // named barrier of the 128 sample threads

template <int MODE>
struct Fmt;
template <>
struct Fmt<DBGZ_PREC_FP32_SPLIT_BF16> {
  static constexpr int NPART = 2, ROWB = 64, ATOM = 512, LAYOUT = 4, NKS = 2, ESZ = 2;
  static constexpr uint32_t IDESC_FMT = 1;  // BF16
};
template <>
struct Fmt<DBGZ_PREC_FP32_TF32> {
  static constexpr int NPART = 1, ROWB = 128, ATOM = 1024, LAYOUT = 2, NKS = 4, ESZ = 4;
  static constexpr uint32_t IDESC_FMT = 2;  // TF32
};

// One problem of a batched launch (global memory): its U^T panel maps and
// the per-problem fields the kernel otherwise takes from UmmaParams.  At most
// two halves (d - 1 <= 256): no re-initialisation, no y workspace.
struct __align__(64) UmmaProb {
  CUtensorMap tm_u[2];
  int64_t d, nY, m, tiles_per_shift;
  dbgz::GenParams gen;
  const float *U32;
  const TargetParams32 *tgt;
  const double *first;  // c1, dc1, up1 of the first dimension (device-computed)
  double *partials;
};

struct __align__(64) UmmaParams {
  CUtensorMap tm_u[2];  // U^T panel parts: rows = targets, K = y-index
  CUtensorMap tm_y[2];  // Y workspace parts: rows = slot*128 + sample, K = y-index
  int64_t d, nY, m, n_reps, tiles_per_shift, n_tiles, tile0;  // tiles [tile0, n_tiles) of the pass
  int P;
  dbgz::GenParams gen;
  const float *U32;  // d x d column-major (in-block triangle)
  const TargetParams32 *tgt;
  double c1, dc1, up1;
  double *partials;
  int *status;
  pol::GradIO<float> io;
  // batched launch: work item `it` is tile item_tile[it] of problem item_prob[it]
  const UmmaProb *probs;
  const int32_t *item_prob, *item_tile;
};

// Block schedule of a tile.  y-block X (X = 0 .. nblk - 1) holds y-indices
// 32X .. 32X + 31, and its targets are those indices + 1.  TMEM holds the
// partial sums of two halves of 128 targets: half h (the targets of blocks
// 4h .. 4h + 3) in columns 128 (h & 1) + 0 .. 127, so that a half's columns
// are free for the half after next as soon as its last block has read them.
constexpr int HB = 4;    // blocks per half
constexpr int HC = 128;  // TMEM columns per half
__device__ __forceinline__ uint32_t tcol(int64_t X) {
  return (uint32_t)(((X >> 2) & 1) * HC + BK * (X & 3));
}
// The last target block that the MMA after block X adds block X's y's to:
// the rest of X's half and the next half, and after the last block of a
// half also the half after that (the first contribution to its columns).
__device__ __forceinline__ int64_t last_target(int64_t X, int64_t nblk) {
  const int64_t h = X >> 2;
  const int64_t e = (X & 3) == 3 ? 4 * h + 11 : 4 * h + 7;
  return e < nblk - 1 ? e : nblk - 1;
}
// Re-initialisation of half g >= 2: the contributions of y-blocks
// 0 .. 4g - 6 to its targets (those of blocks 4g - 5 .. 4g - 1 come from the
// per-block MMAs), as K chunks of one y-block each, issued after the MMAs of
// blocks 4g - 5 .. 4g - 2, a quarter each, while the sample threads work on
// half g - 1.  Block X carries chunks [c0, c1) of half g (empty: c0 == c1).
__device__ __forceinline__ void reinit_share(int64_t X, int64_t nblk, int64_t &g, int64_t &c0, int64_t &c1) {
  g = c0 = c1 = 0;
  if (X < 3) return;
  const int64_t q = (X + 1) & 3;  // X = 4h + 3 + q
  const int64_t h = (X - 3 - q) >> 2;
  if (4 * (h + 2) >= nblk) return;  // no half h + 2
  g = h + 2;
  const int64_t n = 4 * h + 3;
  c0 = q * n / 4;
  c1 = (q + 1) * n / 4;
}

__device__ __forceinline__ void named_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

template <int MODE>
struct Smem {
  static constexpr int ABYTES = TS * Fmt<MODE>::ROWB * Fmt<MODE>::NPART;  // one A tile, all parts
  static constexpr int APART = TS * Fmt<MODE>::ROWB;
  // B stage bytes depend on P: P rows per part
  static __host__ __device__ int bpart(int P) { return P * Fmt<MODE>::ROWB; }
  static __host__ __device__ int bbytes(int P) { return bpart(P) * Fmt<MODE>::NPART; }
  static __host__ __device__ int off_b(int) { return 2 * ABYTES; }
  static __host__ __device__ int off_misc(int P) { return 2 * ABYTES + 2 * bbytes(P); }
  static constexpr int MISC = 15872;  // two CTAs per SM: 2 x (total + 1 KB) <= 228 KB
  static __host__ __device__ int total(int P) { return off_misc(P) + MISC + 1024; }
};

constexpr int kUld = BK + 4;  // row stride of ublk: 16-byte aligned rows for LDS.128
struct Misc {
  // coefficients of the block's triangle, ublk[buf][li][ti] = U[lbase+li, lbase+ti+1], and the
  // block's per-dimension constants; two buffers: the next block stages while this one runs
  float ublk[2][BK][kUld];
  pol::Staged<float> sg[2];
  double red[4];
  // A tiles: a_full (the sample threads wrote a block's y's), a_free (its MMA
  // is done), a_stored (the producer's store of it to the workspace has read
  // it, or it needed none); stages (U^T panels, re-initialisation chunks):
  // b_full, b_free
  uint64_t a_full[2], a_free[2], a_stored[2], b_full[2], b_free[2], bar_s, drain;
  // staging buffers: filled by the producer warp (32 cp.async arrivals when
  // its copies land + 32 arrivals after its own writes), released by the
  // sample threads after the block
  uint64_t stg_full[2], stg_free[2];
  uint32_t tmem_base;
  int abort;
  // Sobol integers of the block's dimensions (dbgz::sobol_stage_block); last,
  // so that kernels that do not stage them are launched without it
  uint32_t sob[2][BK][dbgz::kSobolRow];
};
static_assert(sizeof(Misc) <= Smem<DBGZ_PREC_FP32_TF32>::MISC, "shared scalars exceed their budget");
// dynamic shared memory of a launch: the Sobol staging only where it is used
template <int MODE>
int umma_smem_bytes(int P, bool sobol_staged) {
  return Smem<MODE>::total(P) - (sobol_staged ? 0 : (int)sizeof(Misc::sob));
}

__device__ __forceinline__ void set_abort(Misc *ms, int *status) {
  ms->abort = 1;
  atomicExch(status, DBGZ_ERR_TIMEOUT);
}

// Swizzled K-major offset of 16-byte chunk c of row r.
template <int MODE>
__device__ __forceinline__ uint32_t a_chunk_off(int r, int c) {
  if (MODE == DBGZ_PREC_FP32_SPLIT_BF16)
    return (uint32_t)((r >> 3) * 512 + (r & 7) * 64 + ((c ^ ((r & 7) >> 1)) << 4));
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t t;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(x));
  return t;
}

// s[8 .. 8+N) += sum_k ys[k] * u[k * kUld + 0 .. N), k = 0..7 in order.
template <int N>
__device__ __forceinline__ void rank8_update(float (&s)[BK], const float (&ys)[8], const float *u) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float4 *row = reinterpret_cast<const float4 *>(u + k * kUld);
#pragma unroll
    for (int q = 0; q < N / 4; ++q) {
      const float4 v = row[q];
      s[8 + 4 * q] = fmaf(ys[k], v.x, s[8 + 4 * q]);
      s[9 + 4 * q] = fmaf(ys[k], v.y, s[9 + 4 * q]);
      s[10 + 4 * q] = fmaf(ys[k], v.z, s[10 + 4 * q]);
      s[11 + 4 * q] = fmaf(ys[k], v.w, s[11 + 4 * q]);
    }
  }
}

// Policies that can run a chunk without per-step votes and redo it (Adjoint).
template <typename P, typename = void>
struct chunk_redo : std::false_type {};
template <typename P>
struct chunk_redo<P, std::void_t<decltype(P::kChunkRedo)>> : std::bool_constant<P::kChunkRedo> {};
template <typename P>
constexpr bool chunk_redo_v = chunk_redo<P>::value;

// Policy: pol::Forward<float, GEN, STORE> or pol::Adjoint<float, GEN>.
// BATCH: work items are (problem, tile) pairs of a batched launch, each
// problem at most two halves; every role walks the same static item sequence.
template <int MODE, typename Policy, bool BATCH = false>
__global__ void __launch_bounds__(NT, 2) k_genz_umma(const __grid_constant__ UmmaParams P) {
  using F = Fmt<MODE>;
  using SM = Smem<MODE>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *sm = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *abuf = sm;                       // 2 A tiles
  unsigned char *bst = sm + SM::off_b(P.P);       // 2 B stages
  Misc *ms = reinterpret_cast<Misc *>(sm + SM::off_misc(P.P));
  volatile int *abort = &ms->abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int32_t slot_row = (int32_t)blockIdx.x * TS;  // this CTA's rows of the y workspace
  const int bpart = SM::bpart(P.P);                  // one part of a U^T panel in a stage
  constexpr int kRows = 2 * 64;                      // U^T rows of a re-initialisation chunk
  constexpr int rpart = kRows * F::ROWB;             // one part of its B, after its A
  const uint32_t stage_bytes = (uint32_t)SM::bbytes(P.P);
  static_assert(SM::ABYTES + kRows * F::ROWB * F::NPART <= 256 * F::ROWB * F::NPART,
                "a re-initialisation chunk fills one stage");

  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&ms->a_full[i], 1);
      mbar_init(&ms->a_free[i], 1);
      mbar_init(&ms->a_stored[i], 1);
      mbar_init(&ms->b_full[i], 1);
      mbar_init(&ms->b_free[i], 1);
      mbar_init(&ms->stg_full[i], 64);
      mbar_init(&ms->stg_free[i], 1);
    }
    mbar_init(&ms->bar_s, 1);
    mbar_init(&ms->drain, 1);
    ms->abort = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(&ms->tmem_base, (uint32_t)P.P);
    tmem_relinquish();
  }
  if (!BATCH && warp == kProdWarp && lane == 0) {
    prefetch_tmap(&P.tm_u[0]);
    prefetch_tmap(&P.tm_y[0]);
    if (F::NPART > 1) {
      prefetch_tmap(&P.tm_u[1]);
      prefetch_tmap(&P.tm_y[1]);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = ms->tmem_base;

  if (warp == kProdWarp) {
    // ---------------------------------------------- TMA and block staging
    // Lane 0 issues the TMA traffic: the stage ring (per-block U^T panels
    // and re-initialisation chunks, in the order the MMA warp takes them) and
    // the stores of the y's to the workspace.  All 32 lanes stage each
    // block's U triangle, per-dimension constants and Sobol integers for the
    // sample threads, one block ahead of them (copies by cp.async that arrive
    // on stg_full when they land; stg_free is the sample threads' release of
    // a buffer).
    uint32_t b_use[2] = {0, 0}, jb = 0;
    uint32_t st_use[2] = {0, 0}, st_n = 0;  // stagings per buffer, in all
    bool ok = true;
    int64_t sit = P.tile0 + blockIdx.x, slb = 0;  // the next block to stage: tile, first y-index
    auto stage_next = [&]() -> bool {
      if (sit >= P.n_tiles) return true;
      const int buf = (int)(st_n & 1);
      bool w = true;
      if (st_use[buf] > 0) w = mbar_wait(&ms->stg_free[buf], (st_use[buf] - 1) & 1, abort);
      if (!__all_sync(0xffffffffu, w)) return false;  // the warp decides together
      const UmmaProb *pb = BATCH ? P.probs + P.item_prob[sit] : nullptr;
      const int64_t tile = BATCH ? (int64_t)P.item_tile[sit] : sit;
      const int64_t dI = BATCH ? pb->d : P.d, nYI = BATCH ? pb->nY : P.nY;
      const float *U32I = BATCH ? pb->U32 : P.U32;
      const TargetParams32 *tgtI = BATCH ? pb->tgt : P.tgt;
      Policy pp;
      if (BATCH)
        pp.tile_begin(pb->gen, dI, tile, pb->tiles_per_shift, lane, pb->first[0], pb->first[1], pb->first[2], 0,
                      P.io);
      else
        pp.tile_begin(P.gen, P.d, tile, P.tiles_per_shift, lane, P.c1, P.dc1, P.up1, 0, P.io);
      const int nv = (int)(nYI - slb < BK ? nYI - slb : BK);
      // ublk[li][ti] = U[slb + li, slb + ti + 1] for li <= ti < nv, else 0
#pragma unroll 8
      for (int ti = 0; ti < BK; ++ti) {
        const bool v = lane <= ti && ti < nv;
        pol::cp_async_or_zero<4>(&ms->ublk[buf][lane][ti], v ? U32I + (slb + ti + 1) * dI + slb + lane : U32I, v);
      }
      pp.stage_async(ms->sg[buf], tgtI, lane, slb, nv);
      cp_async_mbar_arrive(&ms->stg_full[buf]);
      mbar_arrive(&ms->stg_full[buf]);
      ++st_use[buf];
      ++st_n;
      slb += BK;
      if (slb >= nYI) {
        slb = 0;
        sit += gridDim.x;
      }
      return true;
    };
    // lane 0: the next stage of the ring (U^T panel or re-initialisation
    // chunk), loaded by `load(stage, full barrier)`
    auto push = [&](auto &&load) -> bool {
      const int ib = (int)(jb & 1);
      if (b_use[ib] > 0 && !mbar_wait(&ms->b_free[ib], (b_use[ib] - 1) & 1, abort)) return false;
      load(bst + ib * stage_bytes, &ms->b_full[ib]);
      ++b_use[ib];
      ++jb;
      return true;
    };
    bool prev_store = false;  // the previous block's y's go to the workspace
    int64_t prev_lb = 0;      // its first y-index
    uint32_t n = 0;           // blocks of this CTA so far
    ok = __all_sync(0xffffffffu, stage_next());  // the CTA's first block
    for (int64_t it = P.tile0 + blockIdx.x; it < P.n_tiles && ok; it += gridDim.x) {
      const UmmaProb *pb = BATCH ? P.probs + P.item_prob[it] : nullptr;
      const CUtensorMap *tmu = BATCH ? pb->tm_u : P.tm_u;
      const int64_t nYi = BATCH ? pb->nY : P.nY;
      const int64_t nblk = (nYi + BK - 1) / BK;
      // later halves are re-initialised from the workspace (halves 0 and 1
      // take every contribution from the per-block MMAs)
      const bool need_ws = !BATCH && nblk > 2 * HB;
      if (BATCH && lane == 0) {
        // the maps were written by a host copy before the launch: order
        // them before the tensor-map proxy reads them (system scope, as the
        // writer is the host)
        for (int pp = 0; pp < F::NPART; ++pp)
          asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(&tmu[pp]) : "memory");
      }
      for (int64_t X = 0; X < nblk && ok; ++X, ++n) {
        // 1. the U^T panel of the MMA after block X: rows of target blocks
        //    X + 1 .. last_target, K = block X's y-indices (the last block of
        //    the tile has no MMA: an empty stage)
        if (lane == 0)
          ok = push([&](unsigned char *st, uint64_t *full) {
            if (X < nblk - 1) {
              const int rows = BK * (int)(last_target(X, nblk) - X);
              const int nbox = (rows + 63) / 64;
              mbar_arrive_expect_tx(full, (uint32_t)(nbox * 64 * F::ROWB * F::NPART));
              for (int pp = 0; pp < F::NPART; ++pp)
                for (int i = 0; i < nbox; ++i)
                  tma_load_2d(st + pp * bpart + i * 64 * F::ROWB, &tmu[pp], (int32_t)(BK * X),
                              (int32_t)(BK * (X + 1) + 1 + 64 * i), full);
            } else {
              mbar_arrive(full);
            }
          });
        ok = __all_sync(0xffffffffu, ok);
        // 2. the staging of the block after this one
        if (ok) ok = __all_sync(0xffffffffu, stage_next());
        if (lane == 0 && ok && n > 0) {
          // 3. the previous block's A tile, once the sample threads are done
          //    with it: its y's to the workspace where a re-initialisation
          //    reads them, then released for reuse
          const int pa = (int)((n - 1) & 1);
          ok = mbar_wait(&ms->a_full[pa], ((n - 1) >> 1) & 1, abort);
          if (ok && prev_store) {
            for (int pp = 0; pp < F::NPART; ++pp)
              tma_store_2d(&P.tm_y[pp], (int32_t)prev_lb, slot_row, abuf + pa * SM::ABYTES + pp * SM::APART);
            bulk_commit();
            bulk_wait_read_all();
          }
          if (ok) mbar_arrive(&ms->a_stored[pa]);
        }
        // y-blocks that a re-initialisation reads: up to 4 g - 6 for the last half g
        prev_store = need_ws && X <= 4 * ((nblk + HB - 1) / HB) - 10;
        prev_lb = BK * X;
        // 4. the re-initialisation chunks carried by block X (the MMA warp
        //    issues them after block X's MMA)
        if (lane == 0 && ok) {
          int64_t g, c0, c1;
          reinit_share(X, nblk, g, c0, c1);
          for (int64_t kc = c0; kc < c1 && ok; ++kc) {
            // y-block kc must be in the workspace: its store is the newest
            // (block X - 1) or an older one
            if (kc == X - 1)
              bulk_wait_all();
            else
              bulk_wait_all_but_1();
            ok = push([&](unsigned char *st, uint64_t *full) {
              mbar_arrive_expect_tx(full, (uint32_t)(SM::ABYTES + kRows * F::ROWB * F::NPART));
              for (int pp = 0; pp < F::NPART; ++pp)
                tma_load_2d(st + pp * SM::APART, &P.tm_y[pp], (int32_t)(BK * kc), slot_row, full);
              for (int pp = 0; pp < F::NPART; ++pp)
                for (int i = 0; i < kRows / 64; ++i)
                  tma_load_2d(st + SM::ABYTES + pp * rpart + i * 64 * F::ROWB, &tmu[pp], (int32_t)(BK * kc),
                              (int32_t)(HC * g + 1 + 64 * i), full);
            });
          }
        }
        ok = __all_sync(0xffffffffu, ok);
      }
    }
    if (!ok && lane == 0) {
      set_abort(ms, P.status);
      // let loads already issued land before the CTA leaves (waits that do
      // not stop at the abort flag, bounded all the same)
      for (int i = 0; i < 2; ++i)
        if (b_use[i] > 0) mbar_wait_drain(&ms->b_full[i], (b_use[i] - 1) & 1);
    }
    if (lane == 0) bulk_wait_all();
    pol::cp_async_wait_all();
  } else if (warp == kMmaWarp) {
    // ---------------------------------------------------------------- MMA
    // Per block X: the MMA of block X's y's into the partial sums of target
    // blocks X + 1 .. last_target (the next block's 32 columns first,
    // committed to bar_s), then the re-initialisation chunks block X carries.
    if (lane == 0) {
      uint32_t a_use[2] = {0, 0}, b_use[2] = {0, 0};
      uint32_t ja = 0, jb = 0;
      bool ok = true;
      const uint32_t sbo = F::ATOM;
      auto issue = [&](uint32_t d_col, int ncols, uint32_t a_addr, uint32_t b_addr, uint32_t b_part, bool overwrite) {
        // D[:, d_col .. d_col+ncols) (+)= A[128 x 32] * B[ncols x 32]^T; split
        // BF16 as hi*hi + hi*lo + lo*hi (parts SM::APART / b_part apart).
        for (int c0 = 0; c0 < ncols; c0 += 256) {
          const int nn = ncols - c0 < 256 ? ncols - c0 : 256;
          const uint32_t idesc = instr_desc(F::IDESC_FMT, F::IDESC_FMT, 128, (uint32_t)nn);
          const uint32_t bo = (uint32_t)(c0 * F::ROWB);
          for (int ks = 0; ks < F::NKS; ++ks) {
            const uint32_t acc0 = (overwrite && ks == 0) ? 0u : 1u;
            const uint64_t a0 = smem_desc(a_addr + 32 * ks, sbo, F::LAYOUT);
            const uint64_t b0 = smem_desc(b_addr + bo + 32 * ks, sbo, F::LAYOUT);
            if (MODE == DBGZ_PREC_FP32_SPLIT_BF16) {
              const uint64_t a1 = smem_desc(a_addr + SM::APART + 32 * ks, sbo, F::LAYOUT);
              const uint64_t b1 = smem_desc(b_addr + b_part + bo + 32 * ks, sbo, F::LAYOUT);
              mma_f16(tmem + d_col + c0, a0, b0, idesc, acc0);
              mma_f16(tmem + d_col + c0, a0, b1, idesc, 1u);
              mma_f16(tmem + d_col + c0, a1, b0, idesc, 1u);
            } else {
              mma_tf32(tmem + d_col + c0, a0, b0, idesc, acc0);
            }
          }
        }
      };
      for (int64_t it = P.tile0 + blockIdx.x; it < P.n_tiles && ok; it += gridDim.x) {
        const int64_t nYi = BATCH ? P.probs[P.item_prob[it]].nY : P.nY;
        const int64_t nblk = (nYi + BK - 1) / BK;
        for (int64_t X = 0; X < nblk && ok; ++X) {
          const int ia = ja & 1, ib = jb & 1;
          ok = mbar_wait(&ms->a_full[ia], a_use[ia] & 1, abort) &&
               mbar_wait(&ms->b_full[ib], b_use[ib] & 1, abort);
          if (!ok) break;
          tc_fence_after();
          if (X < nblk - 1) {
            const uint32_t aa = smem_u32(abuf + ia * SM::ABYTES);
            const uint32_t bb = smem_u32(bst + ib * stage_bytes);
            const int64_t E = last_target(X, nblk), h = X >> 2;
            // the first MMA of a tile writes the columns it touches; the MMA
            // after the last block of half h is the first into half h + 2
            issue(tcol(X + 1), BK, aa, bb, (uint32_t)bpart, X == 0);  // the next block's columns
            mma_commit(&ms->bar_s);
            for (int64_t Y = X + 2; Y <= E;) {
              // target blocks Y .. Ye of one half: contiguous columns
              const int64_t Yh = Y >> 2;
              const int64_t Ye = 4 * Yh + 3 < E ? 4 * Yh + 3 : E;
              issue(tcol(Y), (int)(BK * (Ye - Y + 1)), aa, bb + (uint32_t)(BK * (Y - X - 1) * F::ROWB),
                    (uint32_t)bpart, X == 0 || Yh == h + 2);
              Y = Ye + 1;
            }
            mma_commit(&ms->a_free[ia]);
            mma_commit(&ms->b_free[ib]);
          } else {
            mbar_arrive(&ms->a_free[ia]);
            mbar_arrive(&ms->b_free[ib]);
          }
          ++a_use[ia];
          ++b_use[ib];
          ++ja;
          ++jb;
          // re-initialisation chunks: D = half g's columns, A = y-block kc
          // (from the workspace), B = U^T rows of half g's targets
          int64_t g, c0, c1;
          reinit_share(X, nblk, g, c0, c1);
          const int nbg = (int)(nblk - HB * g < HB ? nblk - HB * g : HB);
          for (int64_t kc = c0; kc < c1 && ok; ++kc) {
            const int ic = jb & 1;
            ok = mbar_wait(&ms->b_full[ic], b_use[ic] & 1, abort);
            if (!ok) break;
            tc_fence_after();
            const uint32_t st = smem_u32(bst + ic * stage_bytes);
            issue((uint32_t)((g & 1) * HC), BK * nbg, st, st + SM::ABYTES, (uint32_t)rpart, false);
            mma_commit(&ms->b_free[ic]);
            ++b_use[ic];
            ++jb;
          }
        }
      }
      if (!ok) set_abort(ms, P.status);
      mma_commit(&ms->drain);
      if (!mbar_wait(&ms->drain, 0, abort)) {
        // abort was raised elsewhere: still give the tensor cores time to finish
        mbar_wait_drain(&ms->drain, 0);
      }
    }
  } else {
    // ------------------------------------------------------ sample threads
    const int r = tid;  // sample row = TMEM lane
    const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
    uint32_t a_use[2] = {0, 0}, ja = 0, s_cnt = 0;
    uint32_t blk = 0;  // blocks run by this CTA (selects the staging buffer)
    for (int64_t it = P.tile0 + blockIdx.x; it < P.n_tiles; it += gridDim.x) {
      const UmmaProb *pb = BATCH ? P.probs + P.item_prob[it] : nullptr;
      const int64_t tile = BATCH ? (int64_t)P.item_tile[it] : it;
      const int64_t dI = BATCH ? pb->d : P.d, nYI = BATCH ? pb->nY : P.nY, mI = BATCH ? pb->m : P.m;
      const int64_t tpsI = BATCH ? pb->tiles_per_shift : P.tiles_per_shift;
      const TargetParams32 *tgtI = BATCH ? pb->tgt : P.tgt;
      double *partsI = BATCH ? pb->partials : P.partials;
      const int64_t nblk = (nYI + BK - 1) / BK;
      const int64_t k_shift = tile / tpsI;
      const int64_t jt = tile - k_shift * tpsI;
      const int64_t j = jt * TS + r;
      Policy pl;
      if (BATCH)
        pl.tile_begin(pb->gen, dI, tile, tpsI, r, pb->first[0], pb->first[1], pb->first[2], 0, P.io);
      else
        pl.tile_begin(P.gen, P.d, tile, P.tiles_per_shift, r, P.c1, P.dc1, P.up1, 0, P.io);
      // this row's terms of the staged Sobol integers of the tile
      const dbgz::SobolLane sob_lane(r, (uint64_t)(pl.gen.sobol_first + pl.gen.gen_base + (pl.j - r)));
      // the Sobol integers of a block's dimensions, staged by the sample
      // threads themselves (warp-wide shuffles, 8 dimensions per warp) into
      // buffer `buf`; visible to all of them after the next block barrier
      const bool sob_staged = Policy::kSobolTable && pl.gen.sobol_staged;
      auto stage_sobol = [&](int buf, int64_t lb) {
        if constexpr (Policy::kSobolTable) {
          const int nv = (int)(nYI - lb < BK ? nYI - lb : BK);
          dbgz::sobol_stage_block(ms->sob[buf], pl.gen.V, pl.gen.ushift + pl.k * (dI - 1),
                                  (uint64_t)(pl.gen.sobol_first + pl.gen.gen_base + (pl.j - r)), pl.sobol_l0(lb),
                                  Policy::kSobolDir, dI - 2, nv, r);
        }
      };
      if (sob_staged) {
        stage_sobol((int)(blk & 1), 0);  // the tile's first block, now
        named_sync(kBarScalar, TS);
      }
      {
        for (int64_t X = 0; X < nblk; ++X) {
          const int ia = ja & 1;
          const int64_t lbase = BK * X;
          const int nval = (int)((nYI - lbase) < BK ? (nYI - lbase) : BK);
          const int cur = (int)(blk & 1);
          // the block's U triangle and per-dimension constants, staged by the
          // producer warp during the previous block
          bool ok = mbar_wait(&ms->stg_full[cur], (blk >> 1) & 1, abort);
          // the next block's Sobol integers while the tensor cores finish this
          // block's partial sums
          if (sob_staged && X + 1 < nblk) stage_sobol(cur ^ 1, lbase + BK);
          float(*ublk)[kUld] = ms->ublk[cur];
          const pol::Staged<float> &sgc = ms->sg[cur];
          // partial sums of the block's targets, accumulated by the tensor cores
          float s[BK];
          if (X == 0) {
#pragma unroll
            for (int t = 0; t < BK; ++t) s[t] = 0.f;
          } else {
            ok = mbar_wait(&ms->bar_s, s_cnt & 1, abort) && ok;
            ++s_cnt;
            tc_fence_after();
            uint32_t v[BK];
            tmem_ld_32x32b_x32(tmem + lane_base + tcol(X), v);
            tmem_wait_ld();
#pragma unroll
            for (int t = 0; t < BK; ++t) s[t] = __uint_as_float(v[t]);
          }
          // the A tile must be free: its previous MMA done, its previous store read
          if (a_use[ia] > 0)
            ok = mbar_wait(&ms->a_free[ia], (a_use[ia] - 1) & 1, abort) &&
                 mbar_wait(&ms->a_stored[ia], (a_use[ia] - 1) & 1, abort) && ok;
          if (!ok) set_abort(ms, P.status);
          // a warp that gives up still meets the others at the block's end,
          // where the decision to leave is taken together
          if (!*abort) {
            // 4 chunks of 8 sequential steps.  s[] is kept in a frame that
            // rotates by 8 per chunk, so that every register index is static:
            // in chunk ch, s[t] is the partial sum of target lbase + 8 ch + t + 1.
            // Step k adds y_k to the chunk's own targets s[k..7] (its
            // triangle); the later chunks' targets s[8 .. 31-8ch] take the
            // chunk's 8 y's in one rank-8 update after the chunk, in the same
            // k order, so every sum is the same fma sequence as step by step.
            unsigned char *A = abuf + ia * SM::ABYTES;
#pragma unroll 1
            for (int ch = 0; ch < BK / 8; ++ch) {
              uint32_t hi[4], lo[4];
              float ys[8];
              pl.chunk_begin(lbase + 8 * ch, nval - 8 * ch);
              // full chunks (all but the last of a problem) run without the
              // per-step bounds test: one uniform branch per chunk instead of 8
              auto steps = [&](auto checked, auto fast) {
#pragma unroll
              for (int k = 0; k < 8; ++k) {
                const int li = 8 * ch + k;
                float y = 0.f;
                if (!decltype(checked)::value || li < nval) {
                  const int64_t l = lbase + li;
                  uint32_t xs = 0u;
                  if constexpr (Policy::kSobolTable)
                    if (pl.gen.sobol_staged) xs = sob_lane.at(ms->sob[cur], li);
                  if constexpr (decltype(fast)::value)
                    y = pl.emit_k_fast(sgc, li, l, k, xs);
                  else
                    y = pl.emit_k(sgc, li, l, k, xs);
                  const float4 *urow = reinterpret_cast<const float4 *>(&ublk[li][8 * ch]);
                  const float4 u0 = urow[0], u1 = urow[1];
                  const float uu[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
                  for (int t = k; t < 8; ++t) s[t] = fmaf(y, uu[t], s[t]);
                  if constexpr (Policy::kDeferTail)
                    pl.consume_deferred(sgc, s[k], li, l, k);
                  else
                    pl.consume(sgc, s[k], li, l);
                }
                ys[k] = y;
              }
              };
              auto run = [&](auto fast) {
                if (nval - 8 * ch >= 8) steps(std::false_type{}, fast);
                else steps(std::true_type{}, fast);
              };
              if constexpr (chunk_redo_v<Policy>) {
                // the chunk without per-step votes; redone with them from its
                // saved state when a lane's FP32 terms left FP32 range
                float s_save[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) s_save[t] = s[t];
                const auto yb_save = pl.ybar;
                pl.bad = false;
                run(std::true_type{});
                if (__any_sync(0xffffffffu, pl.bad)) {
#pragma unroll
                  for (int t = 0; t < 8; ++t) s[t] = s_save[t];
                  pl.ybar = yb_save;
                  pl.fp64_done = 0u;
                  run(std::false_type{});
                }
              } else {
                run(std::false_type{});
              }
              pl.chunk_end(lbase + 8 * ch, nval - 8 * ch);
              if constexpr (Policy::kDeferTail) pl.tail_repair(sgc, s, 8 * ch, lbase + 8 * ch);
              switch (ch) {
                case 0: rank8_update<24>(s, ys, &ublk[0][8]); break;
                case 1: rank8_update<16>(s, ys, &ublk[8][16]); break;
                case 2: rank8_update<8>(s, ys, &ublk[16][24]); break;
                default: break;
              }
              if (MODE == DBGZ_PREC_FP32_SPLIT_BF16) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                  const __nv_bfloat162 h = __floats2bfloat162_rn(ys[2 * e], ys[2 * e + 1]);
                  const float2 hf = __bfloat1622float2(h);
                  hi[e] = *reinterpret_cast<const uint32_t *>(&h);
                  lo[e] = pack_bf16x2(ys[2 * e] - hf.x, ys[2 * e + 1] - hf.y);
                }
                const uint32_t off = a_chunk_off<MODE>(r, ch);
                *reinterpret_cast<uint4 *>(A + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<uint4 *>(A + SM::APART + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
              } else {
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
                  const uint32_t off = a_chunk_off<MODE>(r, 2 * ch + h2);
                  *reinterpret_cast<uint4 *>(A + off) =
                      make_uint4(to_tf32(ys[4 * h2]), to_tf32(ys[4 * h2 + 1]), to_tf32(ys[4 * h2 + 2]),
                                 to_tf32(ys[4 * h2 + 3]));
                }
              }
#pragma unroll
              for (int t = 0; t < BK - 8; ++t) s[t] = s[t + 8];
#pragma unroll
              for (int t = BK - 8; t < BK; ++t) s[t] = 0.f;
            }
          }
          fence_proxy_async_smem();
          tc_fence_before();
          if (bar_red_or(kBarScalar, TS, *abort != 0)) goto done;
          if (r == 0) {
            mbar_arrive(&ms->a_full[ia]);
            mbar_arrive(&ms->stg_free[cur]);
          }
          ++a_use[ia];
          ++ja;
          ++blk;
        }
      }
      // per-tile end and sum of p in a fixed order
      {
        pl.tile_end(tgtI, r, warp, tile, j < mI);
        double pv = pl.tile_value(j < mI);
        for (int o = 16; o > 0; o >>= 1) pv += __shfl_down_sync(0xffffffffu, pv, o);
        if (lane == 0) ms->red[warp] = pv;
        named_sync(kBarScalar, TS);
        if (r == 0) partsI[tile] = ((ms->red[0] + ms->red[1]) + ms->red[2]) + ms->red[3];
      }
    }
  done:;
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, (uint32_t)P.P);
  }
}

// U^T panels: Ut[t * ldU + l] = U[l, t] for l < t (strict upper), else 0.
template <int MODE>
__global__ void k_make_ut(const double *U, int64_t d, int64_t ldU, void *out0, void *out1) {
  const int64_t t = blockIdx.y;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < ldU; l += (int64_t)gridDim.x * blockDim.x) {
    const double u = (l < t && t < d) ? U[t * d + l] : 0.0;
    if (MODE == DBGZ_PREC_FP32_SPLIT_BF16) {
      const __nv_bfloat16 h = __double2bfloat16(u);
      const __nv_bfloat16 lo = __double2bfloat16(u - (double)__bfloat162float(h));
      reinterpret_cast<__nv_bfloat16 *>(out0)[t * ldU + l] = h;
      reinterpret_cast<__nv_bfloat16 *>(out1)[t * ldU + l] = lo;
    } else {
      reinterpret_cast<uint32_t *>(out0)[t * ldU + l] = to_tf32((float)u);
    }
  }
}

typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                            const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                            CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeFn)p;
  }
  return fn;
}

template <int MODE>
int encode_2d(dbgz_ctx *ctx, CUtensorMap *m, void *base, uint64_t inner, uint64_t rows, uint32_t box_rows) {
  using F = Fmt<MODE>;
  EncodeFn enc = encode_fn();
  if (!enc) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[2] = {inner, rows};
  cuuint64_t strides[1] = {inner * F::ESZ};
  cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(m, F::ESZ == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base,
                   dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   F::ESZ == 2 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DBGZ_OK;
}

template <int MODE, int GEN>
auto pick_kind(const PassArgs &pa, bool lower_inf)
    -> decltype(&k_genz_umma<MODE, pol::Forward<float, GEN, false>>) {
  switch (pa.kind) {
    case kLoopForwardStore:
      if (lower_inf) return k_genz_umma<MODE, pol::Forward<float, GEN, true, dbgz::StepFp32LowerInf>>;
      return k_genz_umma<MODE, pol::Forward<float, GEN, true>>;
    case kLoopAdjoint: return k_genz_umma<MODE, pol::Adjoint<float, GEN>>;
    case kLoopLogWeight: return k_genz_umma<MODE, pol::Forward<float, GEN, false, dbgz::StepFp32, true>>;
    default:
      if (lower_inf) return k_genz_umma<MODE, pol::Forward<float, GEN, false, dbgz::StepFp32LowerInf>>;
      return k_genz_umma<MODE, pol::Forward<float, GEN, false>>;
  }
}
template <int MODE>
auto pick_kernel(const PassArgs &pa, bool lower_inf) -> decltype(pick_kind<MODE, 0>(pa, false)) {
  return pa.qmc_type == DBGZ_QMC_SOBOL ? pick_kind<MODE, DBGZ_QMC_SOBOL>(pa, lower_inf)
                                       : pick_kind<MODE, DBGZ_QMC_RICHTMYER>(pa, lower_inf);
}

template <int MODE>
int launch_umma(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  using F = Fmt<MODE>;
  using SM = Smem<MODE>;
  dbgz_ctx *ctx = p->ctx;
  const int64_t d = pa.d, nY = d - 1;
  const int64_t Dp = ((nY + 63) / 64) * 64;
  // converted coefficients (built on first use for this precision): the
  // factor, or its anti-transpose for the adjoint
  const bool adj = pa.kind == kLoopAdjoint;
  if (adj && !p->Ub.p) DBGZ_TRY(dbgz_make_Ub(p));
  DevBuf &src = adj ? p->Ub : p->U;
  DevBuf &u0 = MODE == DBGZ_PREC_FP32_TF32 ? (adj ? p->Ubtf : p->Utf) : (adj ? p->Ubhi : p->Uhi);
  DevBuf &u1 = adj ? p->Ublo : p->Ulo;
  int64_t &ld = adj ? p->ldUb : p->ldU;
  if (!u0.p || ld != Dp || (F::NPART > 1 && !u1.p)) {
    ld = Dp;
    DBGZ_TRY(dbgz_ensure(ctx, u0, (size_t)d * Dp * F::ESZ));
    if (F::NPART > 1) DBGZ_TRY(dbgz_ensure(ctx, u1, (size_t)d * Dp * F::ESZ));
    dim3 g((unsigned)((Dp + 255) / 256), (unsigned)d);
    k_make_ut<MODE><<<g, 256, 0, ctx->stream>>>((const double *)src.p, d, Dp, u0.p,
                                                F::NPART > 1 ? u1.p : nullptr);
    dbgz_count_launch(ctx);
    DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  }
  if (!p->U32.p) DBGZ_TRY(dbgz_make_U32(p));
  const int Pw = 256;
  const int smem = umma_smem_bytes<MODE>(Pw, pa.qmc_type == DBGZ_QMC_SOBOL && !adj);
  auto kern = pick_kernel<MODE>(pa, p->lower_inf);
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  // CTAs per SM from the kernel's own resources: TMEM columns (512 / P),
  // registers and shared memory.  (The runtime occupancy query returns 1 for
  // this kernel although two CTAs fit; if they did not, the extra CTAs would
  // only start later.)
  cudaFuncAttributes fa;
  DBGZ_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, kern));
  int smem_per_sm = 0, regs_per_sm = 0;
  cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device);
  cudaDeviceGetAttribute(&regs_per_sm, cudaDevAttrMaxRegistersPerMultiprocessor, ctx->device);
  const int regs_cta = ((fa.numRegs + 7) / 8) * 8 * NT;
  int per_sm = 512 / Pw;
  per_sm = std::min(per_sm, smem_per_sm / (smem + 1024));
  per_sm = std::min(per_sm, regs_per_sm / std::max(regs_cta, 1));
  if (getenv("DBGZ_DEBUG"))
    fprintf(stderr, "dbgz: tensor-core loop %d CTA/SM (smem %d of %d B, regs %d x %d of %d)\n", per_sm, smem,
            smem_per_sm, fa.numRegs, NT, regs_per_sm);
  if (per_sm < 1) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "tensor-core loop does not fit on an SM");
  const int64_t grid = std::min<int64_t>(n_tiles - pa.tile0, (int64_t)per_sm * ctx->num_sms);
  UmmaParams P{};
  P.d = d;
  P.nY = nY;
  P.m = pa.m;
  P.n_reps = pa.n_reps;
  P.tiles_per_shift = (pa.m + TS - 1) / TS;
  P.n_tiles = n_tiles;
  P.tile0 = pa.tile0;
  P.P = Pw;
  P.gen.qmc_type = pa.qmc_type;
  P.gen.n_bits = pa.n_bits;
  P.gen.gen_base = pa.gen_base;
  P.gen.gen_base_dev = pa.gen_base_dev;
  // Sobol points from the per-block staged integers (forward passes)
  P.gen.sobol_staged = pa.qmc_type == DBGZ_QMC_SOBOL && !adj;
  P.gen.sobol_first = pa.sobol_first;
  P.gen.q = (const double *)p->q.p;
  P.gen.shift64 = (const double *)p->shifts.p;
  P.gen.shift32 = (const float *)p->shifts32.p;
  P.gen.V = (const uint32_t *)p->V.p;
  P.gen.ushift = (const uint64_t *)p->ushifts.p;
  P.U32 = (const float *)(adj ? p->Ub32.p : p->U32.p);
  P.io.N = pa.grad.N;
  P.io.rows = pa.d;
  P.io.y = (float *)pa.grad.y;
  P.io.s = (float *)pa.grad.s;
  P.io.dc = (float *)pa.grad.dc;
  P.io.sbar = (float *)pa.grad.sbar;
  P.io.p = pa.grad.p;
  P.io.ga = pa.grad.ga;
  P.io.gb = pa.grad.gb;
  P.io.gu = pa.grad.gu;
  P.io.dc1 = pa.grad.dc1;
  P.io.tile0 = pa.tile0;
  P.tgt = (const TargetParams32 *)p->tgt32.p;
  P.c1 = pa.c1;
  P.dc1 = pa.dc1;
  P.up1 = 1.0 - pa.c1 - pa.dc1;
  P.partials = partials;
  P.status = ctx->d_status;
  DBGZ_TRY(encode_2d<MODE>(ctx, &P.tm_u[0], u0.p, (uint64_t)Dp, (uint64_t)d, 64));
  if (F::NPART > 1) DBGZ_TRY(encode_2d<MODE>(ctx, &P.tm_u[1], u1.p, (uint64_t)Dp, (uint64_t)d, 64));
  // Y workspace: one 128-row slot per CTA, parts side by side
  const size_t part_bytes = (size_t)grid * TS * Dp * F::ESZ;
  DBGZ_TRY(dbgz_ensure(ctx, p->yws, part_bytes * F::NPART));
  for (int pp = 0; pp < F::NPART; ++pp)
    DBGZ_TRY(encode_2d<MODE>(ctx, &P.tm_y[pp], (char *)p->yws.p + pp * part_bytes, (uint64_t)Dp,
                             (uint64_t)grid * TS, TS));
  if (pa.setup_only) return DBGZ_OK;
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  kern<<<(unsigned)grid, NT, smem, ctx->stream>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

// U^T panels of many problems: problems blockIdx.y + i gridDim.y, factor at
// M + off2[k] (d x d), panel at byte offset pan[k] of out0/out1 with leading
// dimension ldU[k] (rows t = 0..d-1).
template <int MODE>
__global__ void k_make_ut_batch(const double *M, int64_t n, const int64_t *dims, const int64_t *off2,
                                const int64_t *ldU, const int64_t *pan, char *out0, char *out1) {
  for (int64_t k = blockIdx.y; k < n; k += gridDim.y) {
  const int64_t d = dims[k], ld = ldU[k];
  const double *U = M + off2[k];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < d * ld; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = e / ld, l = e - t * ld;
    const double u = (l < t) ? U[t * d + l] : 0.0;
    if (MODE == DBGZ_PREC_FP32_SPLIT_BF16) {
      const __nv_bfloat16 h = __double2bfloat16(u);
      const __nv_bfloat16 lo = __double2bfloat16(u - (double)__bfloat162float(h));
      reinterpret_cast<__nv_bfloat16 *>(out0 + pan[k])[e] = h;
      reinterpret_cast<__nv_bfloat16 *>(out1 + pan[k])[e] = lo;
    } else {
      reinterpret_cast<uint32_t *>(out0 + pan[k])[e] = to_tf32((float)u);
    }
  }
  }
}

template <int MODE, int GEN>
auto batch_kernel() {
  return k_genz_umma<MODE, pol::Forward<float, GEN, false>, true>;
}

template <int MODE>
int setup_umma_batch(dbgz_ctx *ctx, const UmmaBatchArgs &A, UmmaBatchPlan *B) {
  using F = Fmt<MODE>;
  using SM = Smem<MODE>;
  const int Pw = 256;
  const int64_t nsel = (int64_t)A.probs.size();
  // panels and per-problem tables
  std::vector<int64_t> dims(nsel), off2(nsel), ld(nsel), pan(nsel);
  size_t pan_bytes = 0;
  int64_t n_items = 0;
  for (int64_t i = 0; i < nsel; ++i) {
    const int64_t k = A.probs[i], d = A.dims[k];
    if (d - 1 > Pw) return dbgz_fail(ctx, DBGZ_ERR_DIMENSION, "tensor batch: d = %lld needs more than two halves", (long long)d);
    dims[i] = d;
    off2[i] = A.off2[k];
    ld[i] = ((d - 1 + 63) / 64) * 64;
    pan[i] = (int64_t)pan_bytes;
    pan_bytes += (size_t)d * ld[i] * F::ESZ;
    pan_bytes = (pan_bytes + 255) & ~size_t(255);
    n_items += A.tiles_per_shift * A.n_reps;
  }
  if (n_items > INT32_MAX) return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "tensor batch: too many tiles");
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t szTab = al(8 * (size_t)nsel);
  const size_t szDesc = al(sizeof(UmmaProb) * (size_t)nsel), szItems = al(4 * (size_t)n_items);
  DBGZ_TRY(dbgz_ensure(ctx, B->buf, al(pan_bytes) * F::NPART + 4 * szTab + szDesc + 2 * szItems + 1024));
  char *base = (char *)B->buf.p;
  auto take = [&](size_t b) {
    char *r = base;
    base += al(b);
    return r;
  };
  B->pan0 = take(pan_bytes);
  B->pan1 = F::NPART > 1 ? take(pan_bytes) : nullptr;
  B->d_dims = (int64_t *)take(szTab);
  B->d_off2 = (int64_t *)take(szTab);
  B->d_ld = (int64_t *)take(szTab);
  B->d_pan = (int64_t *)take(szTab);
  B->d_desc = take(szDesc);
  B->d_iprob = (int32_t *)take(szItems);
  B->d_itile = (int32_t *)take(szItems);
  B->nsel = nsel;
  B->n_items = n_items;
  B->dM = A.dM;
  // descriptors (maps encoded here, on the host, for the plan's fixed buffers)
  std::vector<UmmaProb> hd(nsel);
  for (int64_t i = 0; i < nsel; ++i) {
    const int64_t k = A.probs[i];
    UmmaProb &D = hd[i];
    std::memset(&D, 0, sizeof(D));
    DBGZ_TRY(encode_2d<MODE>(ctx, &D.tm_u[0], B->pan0 + pan[i], (uint64_t)ld[i], (uint64_t)dims[i], 64));
    if (F::NPART > 1)
      DBGZ_TRY(encode_2d<MODE>(ctx, &D.tm_u[1], B->pan1 + pan[i], (uint64_t)ld[i], (uint64_t)dims[i], 64));
    D.d = dims[i];
    D.nY = dims[i] - 1;
    D.m = A.m;
    D.tiles_per_shift = A.tiles_per_shift;
    D.gen.qmc_type = A.qmc_type;
    D.gen.n_bits = A.n_bits;
    D.gen.gen_base = 0;
    D.gen.sobol_first = A.sobol_first;
    D.gen.q = A.dq;
    D.gen.shift32 = A.dsh32 ? A.dsh32 + A.offs[k] : nullptr;
    D.gen.V = A.dV;
    D.gen.ushift = A.dush ? A.dush + A.offs[k] : nullptr;
    D.gen.sobol_staged = A.qmc_type == DBGZ_QMC_SOBOL;
    D.U32 = A.dU32 + A.off2[k];
    D.tgt = A.dt32 + A.off1[k];
    D.first = A.dfirst + 3 * k;
    D.partials = A.dpart + A.part_off[k];
  }
  // items: every tile of every problem, largest problems first (the caller
  // sorts them), dealt to CTAs round robin
  std::vector<int32_t> ip(n_items), itl(n_items);
  int64_t q = 0;
  for (int64_t i = 0; i < nsel; ++i)
    for (int64_t t = 0; t < A.tiles_per_shift * A.n_reps; ++t, ++q) {
      ip[q] = (int32_t)i;
      itl[q] = (int32_t)t;
    }
  // static tables: uploaded once (pageable sources; the stream is synchronised
  // before the host vectors go out of scope)
  cudaStream_t st = ctx->stream;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_dims, dims.data(), 8 * nsel, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_off2, off2.data(), 8 * nsel, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_ld, ld.data(), 8 * nsel, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_pan, pan.data(), 8 * nsel, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_desc, hd.data(), sizeof(UmmaProb) * nsel, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_iprob, ip.data(), 4 * n_items, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(B->d_itile, itl.data(), 4 * n_items, cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // kernel configuration (attributes set here, outside any stream capture)
  const int smem = umma_smem_bytes<MODE>(Pw, A.qmc_type == DBGZ_QMC_SOBOL);
  auto kern = A.qmc_type == DBGZ_QMC_SOBOL ? batch_kernel<MODE, DBGZ_QMC_SOBOL>()
                                           : batch_kernel<MODE, DBGZ_QMC_RICHTMYER>();
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  cudaFuncAttributes fa;
  DBGZ_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, kern));
  int smem_per_sm = 0, regs_per_sm = 0;
  cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device);
  cudaDeviceGetAttribute(&regs_per_sm, cudaDevAttrMaxRegistersPerMultiprocessor, ctx->device);
  int per_sm = std::min(512 / Pw, smem_per_sm / (smem + 1024));
  per_sm = std::min(per_sm, regs_per_sm / std::max(((fa.numRegs + 7) / 8) * 8 * NT, 1));
  if (per_sm < 1) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "tensor batch: kernel does not fit on an SM");
  B->grid = std::min<int64_t>(n_items, (int64_t)per_sm * ctx->num_sms);
  B->smem = smem;
  return DBGZ_OK;
}

template <int MODE>
int enqueue_umma_batch(UmmaBatchPlan *B) {
  dbgz_ctx *ctx = B->ctx;
  cudaStream_t st = ctx->stream;
  k_make_ut_batch<MODE><<<dim3(8, (unsigned)std::min<int64_t>(B->nsel, 65535)), 256, 0, st>>>(
      B->dM, B->nsel, B->d_dims, B->d_off2, B->d_ld, B->d_pan, B->pan0, B->pan1);
  dbgz_count_launch(ctx);
  UmmaParams P{};
  P.P = 256;
  P.n_tiles = B->n_items;
  P.tile0 = 0;
  P.nY = 1;
  P.status = ctx->d_status;
  P.probs = (const UmmaProb *)B->d_desc;
  P.item_prob = B->d_iprob;
  P.item_tile = B->d_itile;
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  auto kern = B->qmc_type == DBGZ_QMC_SOBOL ? batch_kernel<MODE, DBGZ_QMC_SOBOL>()
                                            : batch_kernel<MODE, DBGZ_QMC_RICHTMYER>();
  kern<<<(unsigned)B->grid, NT, B->smem, st>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

}  // namespace

int dbgz_umma_batch_setup(dbgz_ctx *ctx, int precision, const UmmaBatchArgs &A, UmmaBatchPlan **out) {
  *out = nullptr;
  if (A.probs.empty()) return DBGZ_OK;
  UmmaBatchPlan *B = new UmmaBatchPlan;
  B->ctx = ctx;
  B->mode = precision;
  B->qmc_type = A.qmc_type;
  const int rc = precision == DBGZ_PREC_FP32_SPLIT_BF16 ? setup_umma_batch<DBGZ_PREC_FP32_SPLIT_BF16>(ctx, A, B)
                                                        : setup_umma_batch<DBGZ_PREC_FP32_TF32>(ctx, A, B);
  if (rc != DBGZ_OK) {
    dbgz_umma_batch_free(B);
    return rc;
  }
  *out = B;
  return DBGZ_OK;
}

int dbgz_umma_batch_enqueue(UmmaBatchPlan *B) {
  if (!B) return DBGZ_OK;
  return B->mode == DBGZ_PREC_FP32_SPLIT_BF16 ? enqueue_umma_batch<DBGZ_PREC_FP32_SPLIT_BF16>(B)
                                             : enqueue_umma_batch<DBGZ_PREC_FP32_TF32>(B);
}

void dbgz_umma_batch_free(UmmaBatchPlan *B) {
  if (!B) return;
  dbgz_release(B->buf);
  delete B;
}

int dbgz_loop_umma(dbgz_problem *p, const PassArgs &pa, int precision, double *partials, int64_t n_tiles) {
  if (precision == DBGZ_PREC_FP32_SPLIT_BF16)
    return launch_umma<DBGZ_PREC_FP32_SPLIT_BF16>(p, pa, partials, n_tiles);
  return launch_umma<DBGZ_PREC_FP32_TF32>(p, pa, partials, n_tiles);
}

// loop_simt.cu -- the dense Genz integration loop on CUDA cores.
//
// Replaces qmc_loop!(::QMCData) (reference src/qmc.jl:315-444) and
// qmc_loop!(::QMCData_Distributions) (:485-608).  Two instantiations:
//   T = double, StepFp64: the FP64 path (the reference's Float64 numerics);
//   T = float,  StepFp32: FP32 numerics with the contraction on FP32 cores
//                         (an ablation of the tensor-core path).
//
// Work decomposition (one CTA = one tile of 128 samples = 128 consecutive
// points of one shift; persistent CTAs loop over tiles):
//   * y-indices are processed in groups of G = 64 (targets l+1).  At the
//     start of a group, S[128 x 64] = Y[:, 0:g0] U[0:g0, group targets] is a
//     register-tiled SIMT GEMM over all 256 threads, with Y streamed from
//     this CTA's slot of the Y workspace (global, L2-resident at d <= ~800)
//     and U from global, both staged through shared memory.
//   * inside the group, sub-blocks of 32 y-indices run the sequential step
//     (one thread per sample, genz_step.cuh) with the 32 partial sums of
//     the sub-block in registers; each new y_l updates the remaining sums of
//     its sub-block by a rank-1 update (U broadcast from shared memory).
//   * after sub-block 0, all 256 threads add its 32 y's to the sums of
//     sub-block 1 (128 x 32 x 32 GEMM from shared memory).
//   * p is FP64; per-tile sums go to partials[tile] and a finalize kernel
//     reduces them per shift in a fixed order (deterministic results).
#include "loop_simt_kernels.cuh"
#include <algorithm>

using namespace simt;

namespace {

template <typename T, typename Policy>
int launch_simt(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  dbgz_ctx *ctx = p->ctx;
  const int64_t d = pa.d;
  SimtParams<T> P{};
  P.d = d;
  P.m = pa.m;
  P.n_reps = pa.n_reps;
  P.tiles_per_shift = (pa.m + TS - 1) / TS;
  P.n_tiles = n_tiles;
  P.tile0 = pa.tile0;
  P.Dp = ((d - 1 + G - 1) / G) * G;
  P.gen.qmc_type = pa.qmc_type;
  P.gen.n_bits = pa.n_bits;
  P.gen.gen_base = pa.gen_base;
  P.gen.gen_base_dev = pa.gen_base_dev;
  P.gen.sobol_first = pa.sobol_first;
  // staged Sobol integers (not in the adjoint pass)
  P.gen.sobol_staged = pa.qmc_type == DBGZ_QMC_SOBOL && pa.kind != kLoopAdjoint;
  P.gen.q = (const double *)p->q.p;
  P.gen.shift64 = (const double *)p->shifts.p;
  P.gen.shift32 = (const float *)p->shifts32.p;
  P.gen.V = (const uint32_t *)p->V.p;
  P.gen.ushift = (const uint64_t *)p->ushifts.p;
  P.c1 = pa.c1;
  P.dc1 = pa.dc1;
  P.up1 = 1.0 - pa.c1 - pa.dc1;
  P.cdf_form = pa.cdf_form;
  P.partials = partials;
  const bool adj = pa.kind == kLoopAdjoint;
  if (sizeof(T) == 8) {
    P.U = (const T *)(adj ? p->Ub.p : p->U.p);
    P.tgt = (const typename TgtOf<T>::type *)p->tgt64.p;
  } else {
    P.U = (const T *)(adj ? p->Ub32.p : p->U32.p);
    P.tgt = (const typename TgtOf<T>::type *)p->tgt32.p;
  }
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
  const size_t smem = sizeof(SimtSmem<T>);
  auto kern = k_genz_simt<T, Policy>;
  DBGZ_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  DBGZ_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  if (per_sm < 1) return dbgz_fail(ctx, DBGZ_ERR_CUDA, "simt loop: kernel does not fit on an SM");
  int64_t grid = std::min<int64_t>(n_tiles - pa.tile0, (int64_t)per_sm * ctx->num_sms);
  DBGZ_TRY(dbgz_ensure(ctx, p->yws, sizeof(T) * (size_t)P.Dp * TS * grid));
  P.yws = (T *)p->yws.p;
  if (pa.setup_only) return DBGZ_OK;
  kern<<<(unsigned)grid, NT, smem, ctx->stream>>>(P);
  dbgz_count_launch(ctx);
  DBGZ_CUDA_TRY(ctx, cudaGetLastError());
  return DBGZ_OK;
}

template <typename T, int GEN>
int launch_kind(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  switch (pa.kind) {
    case kLoopForwardStore:
      if (p->lower_inf)
        return launch_simt<T, pol::Forward<T, GEN, true, typename dbgz::StepSel<T, true>::type>>(p, pa, partials,
                                                                                             n_tiles);
      return launch_simt<T, pol::Forward<T, GEN, true>>(p, pa, partials, n_tiles);
    case kLoopAdjoint: return launch_simt<T, pol::Adjoint<T, GEN>>(p, pa, partials, n_tiles);
    case kLoopLogWeight:
      return launch_simt<T, pol::Forward<T, GEN, false, typename pol::StepOf<T>::type, true>>(p, pa, partials,
                                                                                            n_tiles);
    default:
      if (p->lower_inf)
        return launch_simt<T, pol::Forward<T, GEN, false, typename dbgz::StepSel<T, true>::type>>(p, pa, partials,
                                                                                              n_tiles);
      return launch_simt<T, pol::Forward<T, GEN, false>>(p, pa, partials, n_tiles);
  }
}

template <typename T>
int launch_gen(dbgz_problem *p, const PassArgs &pa, double *partials, int64_t n_tiles) {
  if (pa.qmc_type == DBGZ_QMC_SOBOL) return launch_kind<T, DBGZ_QMC_SOBOL>(p, pa, partials, n_tiles);
  return launch_kind<T, DBGZ_QMC_RICHTMYER>(p, pa, partials, n_tiles);
}

}  // namespace

int dbgz_loop_simt(dbgz_problem *p, const PassArgs &pa, int precision, double *partials,
                   int64_t n_tiles) {
  if (precision == DBGZ_PREC_FP64) return launch_gen<double>(p, pa, partials, n_tiles);
  return launch_gen<float>(p, pa, partials, n_tiles);
}

int dbgz_finalize_pass(dbgz_problem *p, const double *partials, int64_t tiles_per_shift,
                       int64_t n_pts0, int64_t m, double *reps) {
  int64_t n_reps = p->opts.n_reps;
  k_finalize<<<(unsigned)((n_reps + 127) / 128), 128, 0, p->ctx->stream>>>(
      partials, tiles_per_shift, n_reps, n_pts0, m, reps);
  dbgz_count_launch(p->ctx);
  DBGZ_CUDA_TRY(p->ctx, cudaGetLastError());
  return DBGZ_OK;
}

int dbgz_loop_tiles_per_shift(int64_t m) { return (int)((m + TS - 1) / TS); }

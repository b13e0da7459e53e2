// driver_graph.cu -- the adaptive loop of qmc_pnorm! (src/qmc.jl:783-850)
// driven on the device.
//
// dbgz_pnorm runs one pass per host iteration: launch, read the running
// means back, form the estimate and 3 SEM on the host, decide whether to run
// another pass (src/qmc.jl:824,835) and advance the point offset
// (next_points!, src/qmc_generators.jl:119-131).  Here the same iterations
// run inside one CUDA graph: a conditional WHILE node whose body is one pass
// -- the loop launch, reading the pass's point offset from device memory --
// followed by k_adaptive_step, which folds the pass into the running means
// (the arithmetic of the per-pass finalize), forms the estimate and 3 SEM
// with the host loop's operations in the host loop's order, advances the
// offset and sets the node's condition.  The host launches the graph once
// per call and reads the result; the results are the host loop's bits.
//
// The graph is kept per problem and precision and rebuilt when a buffer or
// constant it was captured with changes.
#include <cstring>
#include <vector>

#include "internal.cuh"

extern "C" int dbgz_first_dim_cdf(dbgz_problem *p);  // api.cu

namespace {

struct DriverState {
  int64_t gen_base;  // point offset of the next pass (advanced after a pass that is followed by another)
  int64_t npts;      // points per shift so far
  double res, err;
};

// One block of 32 threads.  Shift k: Neumaier sum of its tile sums in tile
// order and the running mean, as simt::k_finalize; then the mean over the
// shifts and 3 * sd (the host loop's sd_ref), in FP64 with explicit
// round-to-nearest operations so that no contraction changes a bit.
__global__ void k_adaptive_step(const double *partials, int64_t tps, int64_t n_reps, int64_t m, double *reps,
                                DriverState *S, int64_t max_pts, double max_abs_err, cudaGraphConditionalHandle h) {
  const int64_t n0 = S->npts;
  for (int64_t k = threadIdx.x; k < n_reps; k += blockDim.x) {
    const double *pk = partials + k * tps;
    double s = 0.0, c = 0.0;
    for (int64_t t = 0; t < tps; ++t) {
      const double x = pk[t];
      const double tt = __dadd_rn(s, x);
      if (fabs(s) >= fabs(x)) c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, tt), x));
      else c = __dadd_rn(c, __dadd_rn(__dsub_rn(x, tt), s));
      s = tt;
    }
    s = __dadd_rn(s, c);
    const double inv_tot = __ddiv_rn(1.0, (double)(n0 + m));
    const double mean_rep = __dmul_rn(s, inv_tot);
    const double old_weight = __dmul_rn((double)n0, inv_tot);
    reps[k] = fma(reps[k], old_weight, mean_rep);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double res = 0.0;
    for (int64_t k = 0; k < n_reps; ++k) res = __dadd_rn(res, reps[k]);
    res = __ddiv_rn(res, (double)n_reps);
    double r = 0.0;
    for (int64_t k = 0; k < n_reps; ++k) {
      const double dd = __dsub_rn(reps[k], res);
      r = __dadd_rn(r, __ddiv_rn(__dmul_rn(dd, dd), (double)n_reps));
    }
    const double e = __dmul_rn(3.0, __dsqrt_rn(__ddiv_rn(r, (double)(n_reps - 1))));
    const int64_t npts = n0 + m;
    S->npts = npts;
    S->res = res;
    S->err = e;
    // another pass while n_pts < max_pts and err > max_abs_err (a NaN error stops)
    const bool more = npts < max_pts && e > max_abs_err;
    if (more) S->gen_base += m;
    cudaGraphSetConditional(h, more ? 1u : 0u);
  }
}

int run_pass(dbgz_problem *p, const PassArgs &pa, int precision, double *partials, int64_t n_tiles) {
  const bool sparse = p->structure == DBGZ_STRUCTURE_SPARSE;
  const bool tensor = !sparse && (precision == DBGZ_PREC_FP32_TF32 || precision == DBGZ_PREC_FP32_SPLIT_BF16);
  if (sparse) return dbgz_loop_sparse(p, pa, precision, partials, n_tiles);
  if (tensor) return dbgz_loop_umma(p, pa, precision, partials, n_tiles);
  return dbgz_loop_simt(p, pa, precision, partials, n_tiles);
}

// Everything a captured pass depends on: buffers (by address), constants
// passed by value, options.
std::vector<uint64_t> signature(const dbgz_problem *p, int precision, const PassArgs &pa) {
  std::vector<uint64_t> s;
  auto addp = [&](const void *x) { s.push_back((uint64_t)(uintptr_t)x); };
  auto addd = [&](double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    s.push_back(u);
  };
  s.push_back((uint64_t)precision);
  addd(pa.c1);
  addd(pa.dc1);
  s.push_back((uint64_t)pa.cdf_form);
  s.push_back((uint64_t)p->structure);
  s.push_back((uint64_t)p->band);
  s.push_back((uint64_t)p->ldU);
  s.push_back((uint64_t)p->opts.m);
  s.push_back((uint64_t)p->opts.n_reps);
  s.push_back((uint64_t)p->opts.max_pts);
  addd(p->opts.max_abs_err);
  const DevBuf *bufs[] = {&p->U,      &p->U32,    &p->Uhi,        &p->Ulo,        &p->Utf,         &p->yws,
                          &p->partials, &p->reps, &p->drv_state, &p->q,          &p->shifts,      &p->shifts32,
                          &p->V,      &p->ushifts, &p->tgt32,     &p->tgt64,      &p->csc_colptr,  &p->csc_row,
                          &p->csc_val64, &p->csc_val32};
  for (const DevBuf *b : bufs) {
    addp(b->p);
    s.push_back((uint64_t)b->bytes);
  }
  return s;
}

void drop_graph(dbgz_problem *p, int i) {
  if (p->drv_exec[i]) cudaGraphExecDestroy(p->drv_exec[i]);
  if (p->drv_graph[i]) cudaGraphDestroy(p->drv_graph[i]);
  p->drv_exec[i] = nullptr;
  p->drv_graph[i] = nullptr;
  p->drv_sig[i].clear();
}

int build_graph(dbgz_problem *p, int precision, const PassArgs &pa, int64_t tps, int64_t n_tiles) {
  dbgz_ctx *ctx = p->ctx;
  cudaStream_t st = ctx->stream;
  cudaStreamCaptureStatus cs;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: the context's stream is being captured");
  cudaGraph_t g = nullptr;
  DBGZ_CUDA_TRY(ctx, cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cudaGraphNode_t node;
  if (cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault) != cudaSuccess) {
    cudaGraphDestroy(g);
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: conditional handle (%s)",
                     cudaGetErrorString(cudaGetLastError()));
  }
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) {
    cudaGraphDestroy(g);
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: conditional node (%s)", cudaGetErrorString(cudaGetLastError()));
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGraphDestroy(g);
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: capture (%s)", cudaGetErrorString(cudaGetLastError()));
  }
  const int64_t lc = ctx->launch_count;
  int rc = run_pass(p, pa, precision, (double *)p->partials.p, n_tiles);
  if (rc == DBGZ_OK) {
    k_adaptive_step<<<1, 32, 0, st>>>((const double *)p->partials.p, tps, p->opts.n_reps, p->opts.m,
                                      (double *)p->reps.p, (DriverState *)p->drv_state.p, p->opts.max_pts,
                                      p->opts.max_abs_err, h);
  }
  ctx->launch_count = lc;
  cudaGraph_t out = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(st, &out);
  cudaGetLastError();
  if (rc == DBGZ_OK && ce != cudaSuccess)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: capture failed (%s)", cudaGetErrorString(ce));
  cudaGraphExec_t exec = nullptr;
  if (rc == DBGZ_OK && cudaGraphInstantiate(&exec, g, 0) != cudaSuccess)
    rc = dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: instantiation failed (%s)",
                   cudaGetErrorString(cudaGetLastError()));
  if (rc != DBGZ_OK) {
    cudaGraphDestroy(g);
    return rc;
  }
  p->drv_graph[precision] = g;
  p->drv_exec[precision] = exec;
  return DBGZ_OK;
}

}  // namespace

void dbgz_drop_graphs(dbgz_problem *p) {
  for (int i = 0; i < 4; ++i) drop_graph(p, i);
}

extern "C" int dbgz_pnorm_graph(dbgz_problem *p, int precision, double *result, double *err, int64_t *n_pts,
                                double *qmc_reps) {
  if (!p || !result || !err || !n_pts) return DBGZ_ERR_INVALID_ARGUMENT;
  dbgz_ctx *ctx = p->ctx;
  if (precision < DBGZ_PREC_FP64 || precision > DBGZ_PREC_FP32_SIMT)
    return dbgz_fail(ctx, DBGZ_ERR_INVALID_ARGUMENT, "pnorm_graph: bad precision %d", precision);
  cudaSetDevice(ctx->device);
  const dbgz_opts &o = p->opts;
  const int64_t n_reps = o.n_reps, m = o.m;
  DBGZ_TRY(dbgz_first_dim_cdf(p));
  if (precision != DBGZ_PREC_FP64 && !p->U32.p) DBGZ_TRY(dbgz_make_U32(p));
  const int64_t tps = (m + 127) / 128;
  const int64_t n_tiles = tps * n_reps;
  DBGZ_TRY(dbgz_ensure(ctx, p->partials, sizeof(double) * n_tiles));
  DBGZ_TRY(dbgz_ensure(ctx, p->reps, sizeof(double) * n_reps));
  DBGZ_TRY(dbgz_ensure(ctx, p->drv_state, sizeof(DriverState)));
  PassArgs pa{};
  pa.d = p->d;
  pa.m = m;
  pa.n_reps = n_reps;
  pa.sobol_first = p->sobol_first;
  pa.n_bits = (int)o.n_bits;
  pa.qmc_type = p->qmc_type;
  pa.cdf_form = p->cdf_form;
  pa.c1 = p->c1;
  pa.dc1 = p->dc1;
  pa.gen_base = p->gen_base;
  pa.gen_base_dev = &((DriverState *)p->drv_state.p)->gen_base;
  // the pass's buffers and operands, made outside the capture
  pa.setup_only = true;
  DBGZ_TRY(run_pass(p, pa, precision, (double *)p->partials.p, n_tiles));
  pa.setup_only = false;
  std::vector<uint64_t> sig = signature(p, precision, pa);
  if (!p->drv_exec[precision] || sig != p->drv_sig[precision]) {
    drop_graph(p, precision);
    DBGZ_TRY(build_graph(p, precision, pa, tps, n_tiles));
    p->drv_sig[precision] = sig;
  }
  cudaStream_t st = ctx->stream;
  const DriverState h0{p->gen_base, 0, 0.0, 0.0};
  const bool prof = ctx->profiling;
  const int64_t launches0 = ctx->launch_count;
  if (prof) cudaEventRecord(ctx->ev[0], st);
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(p->reps.p, 0, sizeof(double) * n_reps, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(p->drv_state.p, &h0, sizeof(h0), cudaMemcpyHostToDevice, st));
  DBGZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
  DBGZ_CUDA_TRY(ctx, cudaGraphLaunch(p->drv_exec[precision], st));
  DriverState hs{};
  std::vector<double> reps(n_reps);
  int dev_status = 0;
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(&hs, p->drv_state.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(reps.data(), p->reps.p, 8 * n_reps, cudaMemcpyDeviceToHost, st));
  DBGZ_CUDA_TRY(ctx, cudaMemcpyAsync(&dev_status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (prof) cudaEventRecord(ctx->ev[1], st);
  if (cudaStreamSynchronize(st) != cudaSuccess)
    return dbgz_fail(ctx, DBGZ_ERR_CUDA, "pnorm_graph: %s", cudaGetErrorString(cudaGetLastError()));
  if (dev_status != 0)
    return dbgz_fail(ctx, DBGZ_ERR_TIMEOUT, "pnorm_graph: a bounded wait in the tensor-core loop gave up (status %d)",
                     dev_status);
  p->gen_base = hs.gen_base;
  const int64_t passes = hs.npts / m;
  dbgz_count_launch(ctx, (int)(2 * passes));
  if (prof) {
    dbgz_profile pr{};
    pr.prepare_ms = ctx->prof.prepare_ms;
    pr.prepare_launches = ctx->prof.prepare_launches;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]) == cudaSuccess) pr.pnorm_ms = ms;
    pr.loop_launches = passes;
    pr.kernel_launches = ctx->launch_count - launches0;
    ctx->prof = pr;
  }
  *result = hs.res;
  *err = hs.err;
  *n_pts = hs.npts;
  if (qmc_reps) std::memcpy(qmc_reps, reps.data(), sizeof(double) * n_reps);
  return DBGZ_OK;
}

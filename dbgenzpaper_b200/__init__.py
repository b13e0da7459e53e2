"""dbgenzpaper_b200 -- B200-native Genz QMC multivariate-normal probabilities.

Host-side mirror of the reference package's API (JakobPeterlin/DBGenzPaper,
src/DBGenzPaper.jl exports) over the C ABI of ``libdbgenz.so``:

====================================  =====================================
reference (Julia)                     here
====================================  =====================================
``QMC_opts(T; kw...)`` qmc.jl:111     ``QMC_opts(T, **kw)``
``QMCData(C,a,b,opts,rng,type)``      ``QMCData(C, a, b, opts, rng, type)``
``QMCDataSparse(...)`` qmc.jl:225     ``QMCDataSparse(...)``
``QMCData_Distributions(D)`` :210     ``QMCData_Distributions(D)``
``qmc_pnorm!(D)`` qmc.jl:783          ``qmc_pnorm(D)``
``cholesky_genz!`` cholesky.jl:445    ``cholesky_genz(M, a, b, ...)``
``cholesky_classic!`` :144            ``cholesky_classic(M, a, b, ...)``
``get_sqrt_primes!`` generators:300   ``get_sqrt_primes(n)``
``richtmyer_mat!`` generators:314     ``richtmyer_mat(m, q, n0)``
``sobol_mat!`` generators:331         ``sobol_mat(m, V, first)``
====================================  =====================================

Everything computes on the GPU; there is no CPU path.  The working type ``T``
of ``QMC_opts`` selects the precision: ``np.float64`` runs the FP64 kernels,
``np.float32`` the mixed-precision ones (FP32 special functions, FP64 weight
product and reductions, tensor-core contraction).  A ``precision=`` keyword
picks any mode of ``dbgz_precision`` explicitly.

Random shifts: the reference draws them from a Julia RNG inside the
constructor (``rand(rng, T, n-1, n_reps)``); here ``rng`` is a numpy
``Generator`` (or the shifts are passed explicitly with ``shifts=``), since
Julia's stream cannot be reproduced outside Julia.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from typing import NamedTuple, Optional

import numpy as np

from . import _lib as L

__all__ = [
    "QMCOpts", "QMC_opts", "QMCData", "QMCDataSparse", "QMCData_Distributions",
    "qmc_pnorm", "qmc_pnorm_grad", "qmc_pnorm_logw", "log_mean_exp", "CholeskyGenz", "cholesky_genz",
    "cholesky_classic", "cholesky_rowmax", "adapt_low_rank", "sobol_first_index",
    "get_sqrt_primes", "richtmyer_mat", "sobol_mat", "sobol_dirnums", "Context",
    "get_context", "DbgzError", "PRECISIONS", "qmc_pnorm_batch", "BatchPlan", "batch_autotune",
    "batch_tuning",
]

DbgzError = L.DbgzError
PRECISIONS = {
    "fp64": L.PREC_FP64,
    "fp32_tf32": L.PREC_FP32_TF32,
    "fp32_split_bf16": L.PREC_FP32_SPLIT_BF16,
    "fp32_simt": L.PREC_FP32_SIMT,
}
# precision used for QMC_opts(np.float32)
DEFAULT_FP32_PRECISION = L.PREC_FP32_SPLIT_BF16


class Context:
    """One CUDA device and stream of libdbgenz (dbgz_create/dbgz_destroy)."""

    def __init__(self, device: int = 0):
        self._lib = L.lib()
        h = C.c_void_p()
        L.check(self._lib.dbgz_create(int(device), C.byref(h)))
        self.handle = h
        self.device = device

    def release_cached(self) -> int:
        """Return the context's cached device buffers to the driver; -> bytes freed."""
        n = C.c_uint64()
        L.check(self._lib.dbgz_release_cached(self.handle, C.byref(n)), self.handle)
        return int(n.value)

    def set_state_budget(self, nbytes: int) -> None:
        """Cap the device memory of stored forward state in gradient calls
        (larger sample counts run in chunks of tiles)."""
        L.check(self._lib.dbgz_set_state_budget(self.handle, int(nbytes)), self.handle)

    def set_grad_checkpoints(self, segment: int) -> None:
        """Banded gradients: a checkpoint every `segment` dimensions, each
        segment recomputed from its checkpoint before the adjoint sweeps it
        (default 256; 0 stores the whole forward state).  Same results."""
        L.check(self._lib.dbgz_set_grad_checkpoints(self.handle, int(segment)), self.handle)

    def close(self):
        if self.handle:
            if self._lib.dbgz_destroy(self.handle) == L.OK:
                self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}


def get_context(device: int = 0) -> Context:
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = _contexts[device] = Context(device)
    return ctx


# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class QMCOpts:
    """QMCOpts{T} (src/qmc.jl:15-27)."""
    T: type
    chol_block_size: int
    chol_block_size2: int
    m: int
    block_size_i: int
    block_size_i2: int
    block_size_j: int
    n_blocks: int
    n_reps: int
    n_bits: int
    max_pts: int
    max_abs_err: float

    def to_c(self) -> L.DbgzOpts:
        return L.DbgzOpts(self.chol_block_size, self.chol_block_size2, self.m,
                          self.block_size_i, self.block_size_i2, self.block_size_j,
                          self.n_blocks, self.n_reps, self.n_bits, self.max_pts,
                          float(self.max_abs_err))


def QMC_opts(T=np.float64, *, chol_block_size=2**6, chol_block_size2=2**9, m=10**4,
             block_size_i=2**6, block_size_j=2**6, block_size_i2=2**5, n_blocks=1,
             n_reps=12, n_bits=32, max_pts=10**4, max_abs_err=1e-6) -> QMCOpts:
    """QMC_opts(T; ...) with the reference's defaults (src/qmc.jl:111-125)."""
    T = np.dtype(T).type
    if T not in (np.float64, np.float32):
        raise TypeError("T must be float64 or float32")
    return QMCOpts(T, int(chol_block_size), int(chol_block_size2), int(m), int(block_size_i),
                   int(block_size_i2), int(block_size_j), int(n_blocks), int(n_reps),
                   int(n_bits), int(max_pts), float(max_abs_err))


class CholeskyGenz(NamedTuple):
    """CholeskyGenz{T} (src/cholesky.jl:5-14); perm is 0-based."""
    U: np.ndarray
    perm: np.ndarray
    rank: int
    a: np.ndarray
    b: np.ndarray
    block_size: int
    pivot_method: str
    scale_vec: np.ndarray


def _f64(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


# ---------------------------------------------------------------------------
class QMCData:
    """QMCData (src/qmc.jl:149-202): factorisation, generator and workspaces
    of one problem, resident on the GPU."""

    _structure = L.STRUCTURE_DENSE
    _default_type = "Richtmyer"

    def __init__(self, C_mat, a, b, opts: Optional[QMCOpts] = None, rng=None, qmc_type=None, *,
                 shifts=None, ushifts=None, sobol_dirnums=None, sobol_first=None,
                 precision: Optional[int] = None, cdf_form: int = L.CDF_ERF, device: int = 0,
                 context: Optional[Context] = None):
        qmc_type = self._default_type if qmc_type is None else str(qmc_type).lstrip(":")
        if qmc_type not in ("Richtmyer", "Sobol"):
            raise ValueError("qmc_type must be 'Richtmyer' or 'Sobol'")
        opts = QMC_opts() if opts is None else opts
        Sig = np.asfortranarray(np.asarray(C_mat, dtype=np.float64))
        n = Sig.shape[0]
        if Sig.shape != (n, n):
            raise ValueError("C must be square")
        a, b = _f64(a), _f64(b)
        if a.shape != (n,) or b.shape != (n,):
            raise ValueError("a and b must have length n")
        rng = np.random.default_rng() if rng is None else rng
        self.ctx = get_context(device) if context is None else context
        self.n = n
        self.opts = opts
        self.qmc_type = qmc_type
        self.precision = precision
        self.cdf_form = cdf_form
        d1 = max(n - 1, 1)
        sh = ush = V = None
        first = 0
        if qmc_type == "Richtmyer":
            sh = rng.random((d1, opts.n_reps)) if shifts is None else np.asarray(shifts, np.float64)
            if opts.T == np.float32 and shifts is None:
                sh = sh.astype(np.float32).astype(np.float64)
            sh = np.asfortranarray(sh)
            if sh.shape != (d1, opts.n_reps):
                raise ValueError(f"shifts must be {(d1, opts.n_reps)}")
        else:
            if ushifts is None:
                ush = rng.integers(0, 2**64, size=(d1, opts.n_reps), dtype=np.uint64, endpoint=False)
            else:
                ush = np.asarray(ushifts, dtype=np.uint64)
            ush = np.asfortranarray(ush)
            if sobol_dirnums is not None:
                V = np.ascontiguousarray(sobol_dirnums, dtype=np.uint32)
            first = sobol_first_index(opts.m) if sobol_first is None else int(sobol_first)
        self.shifts, self.ushifts, self.sobol_dirnums, self.sobol_first = sh, ush, V, first
        h = C.c_void_p()
        co = opts.to_c()
        st = L.lib().dbgz_prepare(self.ctx.handle, n, L.ptr(Sig), L.ptr(a), L.ptr(b), C.byref(co),
                                  L.QMC_RICHTMYER if qmc_type == "Richtmyer" else L.QMC_SOBOL,
                                  self._structure, int(cdf_form), L.ptr(sh),
                                  L.ptr(ush, C.c_uint64), L.ptr(V, C.c_uint32), first, C.byref(h))
        L.check(st, self.ctx.handle)
        self.handle = h
        self._chol = None

    @property
    def C(self) -> CholeskyGenz:
        if self._chol is None:
            n = self.n
            U = np.zeros((n, n), order="F")
            perm = np.zeros(n, dtype=np.int64)
            a, b, sv = np.zeros(n), np.zeros(n), np.zeros(n)
            rank = C.c_int64()
            L.check(L.lib().dbgz_problem_factor(self.handle, L.ptr(U), L.ptr(perm, C.c_int64),
                                                L.ptr(a), L.ptr(b), L.ptr(sv), C.byref(rank)),
                    self.ctx.handle)
            method = "genz" if self._structure == L.STRUCTURE_DENSE else "none"
            self._chol = CholeskyGenz(U, perm, rank.value, a, b, self.opts.chol_block_size,
                                      method, sv)
        return self._chol

    def truncate_band(self, bandwidth: int) -> None:
        """Drop factor entries more than `bandwidth` above the diagonal (the
        banded workload's truncation; no counterpart in the reference)."""
        L.check(L.lib().dbgz_problem_truncate_band(self.handle, int(bandwidth)), self.ctx.handle)
        self._chol = None

    @property
    def a(self):
        return self.C.a

    @property
    def b(self):
        return self.C.b

    def resolved_precision(self) -> int:
        if self.precision is not None:
            return int(self.precision)
        return L.PREC_FP64 if self.opts.T == np.float64 else DEFAULT_FP32_PRECISION

    def close(self):
        if getattr(self, "handle", None):
            L.lib().dbgz_problem_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class QMCDataSparse(QMCData):
    """QMCDataSparse (src/qmc.jl:225-282): classic (unpivoted) Cholesky and
    the loop over the strict-upper CSC of U.  Default generator: Sobol."""

    _structure = L.STRUCTURE_SPARSE
    _default_type = "Sobol"


class QMCData_Distributions:
    """QMCData_Distributions(D) (src/qmc.jl:210-215): the same problem and
    generator state as D, integrated with the erfc form of the CDF."""

    def __init__(self, D: QMCData):
        self.D = D

    def __getattr__(self, name):
        return getattr(self.D, name)


def qmc_pnorm(D, use_AppleBLAS=None, *, precision: Optional[int] = None, return_reps=False,
              driver: str = "host"):
    """qmc_pnorm!(D) (src/qmc.jl:783-850) -> (result, err, n_pts).

    ``use_AppleBLAS`` is accepted for signature compatibility (it only steers
    CPU BLAS threading in the reference).  With ``return_reps`` the per-shift
    running means are returned as a fourth element.  ``driver="graph"`` runs
    the adaptive loop on the device (dbgz_pnorm_graph: one CUDA graph launch
    for all passes); the results are the same bits."""
    if driver not in ("host", "graph"):
        raise ValueError("driver must be 'host' or 'graph'")
    dist = isinstance(D, QMCData_Distributions)
    base = D.D if dist else D
    prec = base.resolved_precision() if precision is None else int(precision)
    res, err, npts = C.c_double(), C.c_double(), C.c_int64()
    reps = np.zeros(base.opts.n_reps)
    lib = L.lib()
    if dist:
        lib.dbgz_problem_set_cdf_form(base.handle, L.CDF_ERFC)
    try:
        fn = lib.dbgz_pnorm_graph if driver == "graph" else lib.dbgz_pnorm
        st = fn(base.handle, prec, C.byref(res), C.byref(err), C.byref(npts), L.ptr(reps))
    finally:
        if dist:
            lib.dbgz_problem_set_cdf_form(base.handle, int(base.cdf_form))
    L.check(st, base.ctx.handle)
    out = (res.value, err.value, int(npts.value))
    return out + (reps,) if return_reps else out


def qmc_pnorm_logw(D, *, precision: Optional[int] = None):
    """Per-sample log-weights of one pass (dbgz_pnorm_logw; no reference
    counterpart) -> (logw, reps): logw[j, k] = log p of point j of shift k,
    the sum of log dc over the sample's variables, finite where p underflows;
    reps the pass's per-shift means of p.  The pass uses the points the next
    qmc_pnorm pass would take and does not advance the generator."""
    dist = isinstance(D, QMCData_Distributions)
    base = D.D if dist else D
    prec = base.resolved_precision() if precision is None else int(precision)
    m, R = base.opts.m, base.opts.n_reps
    logw = np.zeros((m, R), dtype=np.float64, order="F")
    reps = np.zeros(R)
    lib = L.lib()
    if dist:
        lib.dbgz_problem_set_cdf_form(base.handle, L.CDF_ERFC)
    try:
        st = lib.dbgz_pnorm_logw(base.handle, prec, L.ptr(logw), L.ptr(reps))
    finally:
        if dist:
            lib.dbgz_problem_set_cdf_form(base.handle, int(base.cdf_form))
    L.check(st, base.ctx.handle)
    return logw, reps


def log_mean_exp(logw, axis=0):
    """log of the mean of exp(logw) along axis, without underflow: the log of
    the per-shift estimate from per-sample log-weights."""
    x = np.asarray(logw, dtype=np.float64)
    mx = np.max(x, axis=axis, keepdims=True)
    mx = np.where(np.isfinite(mx), mx, 0.0)
    return np.squeeze(mx, axis=axis) + np.log(np.mean(np.exp(x - mx), axis=axis))


def qmc_pnorm_grad(D, *, precision: Optional[int] = None, want_U: bool = True):
    """Estimate and exact gradient on the current point set (no counterpart
    in the reference): -> (P, err, n_pts, dP_da, dP_db, dP_dU).

    dP_da/dP_db are in the original variable order and scale; dP_dU is with
    respect to the factor in the permuted, scaled coordinates of ``D.C``."""
    base = D.D if isinstance(D, QMCData_Distributions) else D
    prec = base.resolved_precision() if precision is None else int(precision)
    n = base.n
    res, err, npts = C.c_double(), C.c_double(), C.c_int64()
    da, db = np.zeros(n), np.zeros(n)
    want_U = want_U and base._structure == L.STRUCTURE_DENSE  # the banded path gives da, db only
    dU = np.zeros((n, n), order="F") if want_U else None
    L.check(L.lib().dbgz_pnorm_grad(base.handle, prec, C.byref(res), C.byref(err), C.byref(npts), L.ptr(da),
                                    L.ptr(db), L.ptr(dU)), base.ctx.handle)
    return res.value, err.value, int(npts.value), da, db, dU


def sigma_adjoint(D, dP_dU, dP_da=None, dP_db=None) -> np.ndarray:
    """dP/dSigma (original order, symmetric; dP = sum_ij G_ij E_ij for a
    symmetric perturbation E) from the outputs of qmc_pnorm_grad, through
    the pivoted Cholesky (permutation held fixed) and the correlation scaling
    (no counterpart in the reference).  For Sigma = B B' + diag(psi):
    dP/dB = 2 G B."""
    base = D.D if isinstance(D, QMCData_Distributions) else D
    n = base.n
    G = np.zeros((n, n), order="F")
    dU = np.asfortranarray(np.asarray(dP_dU, dtype=np.float64))
    da = None if dP_da is None else _f64(dP_da)
    db = None if dP_db is None else _f64(dP_db)
    L.check(L.lib().dbgz_problem_sigma_adjoint(base.handle, L.ptr(dU), L.ptr(da), L.ptr(db), L.ptr(G)),
            base.ctx.handle)
    return G


def qmc_pnorm_grad_sigma(D, *, precision: Optional[int] = None):
    """Estimate and gradients with respect to the inputs of QMCData, the
    factor gradient kept on the device (dbgz_pnorm_grad_sigma):
    -> (P, err, n_pts, dP_da, dP_db, dP_dSigma), all in the original order."""
    base = D.D if isinstance(D, QMCData_Distributions) else D
    prec = base.resolved_precision() if precision is None else int(precision)
    n = base.n
    res, err, npts = C.c_double(), C.c_double(), C.c_int64()
    da, db = np.zeros(n), np.zeros(n)
    G = np.zeros((n, n), order="F")
    L.check(L.lib().dbgz_pnorm_grad_sigma(base.handle, prec, C.byref(res), C.byref(err), C.byref(npts),
                                          L.ptr(da), L.ptr(db), L.ptr(G)), base.ctx.handle)
    return res.value, err.value, int(npts.value), da, db, G


def qmc_pnorm_batch(problems, opts: Optional[QMCOpts] = None, rng=None, qmc_type="Richtmyer", *,
                    shifts=None, ushifts=None, sobol_dirnums=None, sobol_first=None,
                    precision: Optional[int] = None, device: int = 0, context: Optional[Context] = None,
                    return_ranks: bool = False):
    """P and 3 SEM of many independent problems in one call (dbgz_pnorm_batch;
    no counterpart in the reference, which loops over QMCData/qmc_pnorm!).

    problems: sequence of (Sigma, a, b).  One pass of opts.m points x
    opts.n_reps shifts per problem.  shifts / ushifts: sequences of the
    per-problem (d-1, n_reps) arrays (drawn from rng when None).  Returns
    (P, err) arrays (and the ranks with return_ranks); a problem that is not
    full rank raises, unless return_ranks is set (its P is then NaN)."""
    qmc_type = str(qmc_type).lstrip(":")
    if qmc_type not in ("Richtmyer", "Sobol"):
        raise ValueError("qmc_type must be 'Richtmyer' or 'Sobol'")
    opts = QMC_opts() if opts is None else opts
    rng = np.random.default_rng() if rng is None else rng
    ctx = get_context(device) if context is None else context
    dims = np.array([np.asarray(p[0]).shape[0] for p in problems], dtype=np.int64)
    Sig = np.concatenate([np.ravel(np.asarray(p[0], dtype=np.float64), order="F") for p in problems])
    a = np.concatenate([_f64(p[1]) for p in problems])
    b = np.concatenate([_f64(p[2]) for p in problems])
    R = opts.n_reps
    sh = ush = V = None
    first = 0
    if qmc_type == "Richtmyer":
        if shifts is None:
            shifts = [rng.random((d - 1, R)) for d in dims]
        sh = np.concatenate([np.ravel(np.asarray(x, dtype=np.float64), order="F") for x in shifts])
    else:
        if ushifts is None:
            ushifts = [rng.integers(0, 2**64, size=(d - 1, R), dtype=np.uint64, endpoint=False) for d in dims]
        ush = np.concatenate([np.ravel(np.asarray(x, dtype=np.uint64), order="F") for x in ushifts])
        if sobol_dirnums is not None:
            V = np.ascontiguousarray(sobol_dirnums, dtype=np.uint32)
        first = sobol_first_index(opts.m) if sobol_first is None else int(sobol_first)
    prec = (L.PREC_FP64 if opts.T == np.float64 else DEFAULT_FP32_PRECISION) if precision is None else int(precision)
    n = len(problems)
    P, err = np.zeros(n), np.zeros(n)
    ranks = np.zeros(n, dtype=np.int64)
    co = opts.to_c()
    st = L.lib().dbgz_pnorm_batch(ctx.handle, n, L.ptr(dims, C.c_int64), L.ptr(Sig), L.ptr(a), L.ptr(b),
                                  C.byref(co), L.QMC_RICHTMYER if qmc_type == "Richtmyer" else L.QMC_SOBOL,
                                  prec, L.ptr(sh), L.ptr(ush, C.c_uint64), L.ptr(V, C.c_uint32), first,
                                  L.ptr(P), L.ptr(err), L.ptr(ranks, C.c_int64))
    if return_ranks and st == L.ERR_RANK_DEFICIENT:
        return P, err, ranks
    L.check(st, ctx.handle)
    return (P, err, ranks) if return_ranks else (P, err)


class BatchPlan:
    """A reusable batch (dbgz_batch_plan_*; no counterpart in the reference):
    the problems' dimensions, options, generator and precision are fixed at
    creation, which makes the device buffers, tensor maps and a CUDA graph of
    one run.  Fill the plan's pinned host buffers -- `fill(problems, ...)`,
    or write the packed numpy views `Sigma`, `a`, `b`, `shifts` directly --
    then `run()`: one graph launch uploads them, checks them, factorises,
    integrates, reduces and reads back.  Richtmyer shifts are doubles in
    [0, 1], Sobol shifts uint64 digital shifts."""

    def __init__(self, dims, opts: Optional[QMCOpts] = None, qmc_type="Richtmyer", *,
                 precision: Optional[int] = None, sobol_dirnums=None, sobol_first=None,
                 device: int = 0, context: Optional[Context] = None):
        qmc_type = str(qmc_type).lstrip(":")
        if qmc_type not in ("Richtmyer", "Sobol"):
            raise ValueError("qmc_type must be 'Richtmyer' or 'Sobol'")
        self.opts = QMC_opts() if opts is None else opts
        self.qmc_type = qmc_type
        self.ctx = get_context(device) if context is None else context
        self.dims = np.ascontiguousarray(dims, dtype=np.int64)
        R = self.opts.n_reps
        self.precision = ((L.PREC_FP64 if self.opts.T == np.float64 else DEFAULT_FP32_PRECISION)
                          if precision is None else int(precision))
        V = None if sobol_dirnums is None else np.ascontiguousarray(sobol_dirnums, dtype=np.uint32)
        first = sobol_first_index(self.opts.m) if sobol_first is None else int(sobol_first)
        self._lib = L.lib()
        h = C.c_void_p()
        co = self.opts.to_c()
        L.check(self._lib.dbgz_batch_plan_create(
            self.ctx.handle, len(self.dims), L.ptr(self.dims, C.c_int64), C.byref(co),
            L.QMC_RICHTMYER if qmc_type == "Richtmyer" else L.QMC_SOBOL, self.precision,
            L.ptr(V, C.c_uint32), first, C.byref(h)), self.ctx.handle)
        self.handle = h
        pS, pa, pb, psh = L._pd(), L._pd(), L._pd(), C.c_void_p()
        L.check(self._lib.dbgz_batch_plan_buffers(h, C.byref(pS), C.byref(pa), C.byref(pb), C.byref(psh)))
        d = self.dims
        s2, s1, ss = int((d * d).sum()), int(d.sum()), int(((d - 1) * R).sum())
        self.off2 = np.concatenate([[0], np.cumsum(d * d)[:-1]]).astype(np.int64)
        self.off1 = np.concatenate([[0], np.cumsum(d)[:-1]]).astype(np.int64)
        self.offs = np.concatenate([[0], np.cumsum((d - 1) * R)[:-1]]).astype(np.int64)
        self.Sigma = np.ctypeslib.as_array(pS, shape=(s2,))
        self.a = np.ctypeslib.as_array(pa, shape=(s1,))
        self.b = np.ctypeslib.as_array(pb, shape=(s1,))
        sht = C.c_double if qmc_type == "Richtmyer" else C.c_uint64
        self.shifts = np.ctypeslib.as_array(C.cast(psh, C.POINTER(sht)), shape=(ss,))

    def set_problem(self, k: int, Sigma, a, b, shifts) -> None:
        """Write problem k's Sigma (d x d), bounds and (d-1, n_reps) shifts."""
        d = int(self.dims[k])
        R = self.opts.n_reps
        self.Sigma[self.off2[k]:self.off2[k] + d * d] = np.ravel(np.asarray(Sigma, dtype=np.float64), order="F")
        self.a[self.off1[k]:self.off1[k] + d] = _f64(a)
        self.b[self.off1[k]:self.off1[k] + d] = _f64(b)
        self.shifts[self.offs[k]:self.offs[k] + (d - 1) * R] = np.ravel(
            np.asarray(shifts, dtype=self.shifts.dtype), order="F")

    def fill(self, problems, shifts) -> None:
        """problems: sequence of (Sigma, a, b); shifts: the per-problem (d-1, n_reps) arrays."""
        for k, (S, a, b) in enumerate(problems):
            self.set_problem(k, S, a, b, shifts[k])

    def run(self, return_ranks: bool = False):
        """One graph launch; -> (P, err) (and the ranks with return_ranks)."""
        n = len(self.dims)
        P, err = np.zeros(n), np.zeros(n)
        ranks = np.zeros(n, dtype=np.int64)
        st = self._lib.dbgz_batch_plan_run(self.handle, L.ptr(P), L.ptr(err), L.ptr(ranks, C.c_int64))
        if return_ranks and st == L.ERR_RANK_DEFICIENT:
            return P, err, ranks
        L.check(st, self.ctx.handle)
        return (P, err, ranks) if return_ranks else (P, err)

    def info(self) -> dict:
        """Tensor-core problems, SIMT work items, kernels per run, pinned input bytes."""
        v = [C.c_int64() for _ in range(4)]
        L.check(self._lib.dbgz_batch_plan_info(self.handle, *[C.byref(x) for x in v]))
        return dict(zip(("tensor_problems", "simt_items", "kernels_per_run", "host_bytes"),
                        [int(x.value) for x in v]))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.dbgz_batch_plan_destroy(self.handle)
            self.handle = None
            self.Sigma = self.a = self.b = self.shifts = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(opts: Optional[QMCOpts] = None, precision: Optional[int] = None, qmc_type="Sobol", *,
                   device: int = 0, context: Optional[Context] = None):
    """dbgz_batch_autotune: time the batch loops per dimension bucket on pilot
    batches of opts' point and shift counts and keep the fastest choice in
    the context.  -> (engine, item_dims), arrays indexed by d = 0..512
    (engine 1 = tensor-core loop, 0 = SIMT loop)."""
    opts = QMC_opts() if opts is None else opts
    ctx = get_context(device) if context is None else context
    prec = ((L.PREC_FP64 if opts.T == np.float64 else DEFAULT_FP32_PRECISION)
            if precision is None else int(precision))
    qmc_type = str(qmc_type).lstrip(":")
    eng = np.zeros(513, dtype=np.int32)
    items = np.zeros(513, dtype=np.int32)
    co = opts.to_c()
    L.check(L.lib().dbgz_batch_autotune(ctx.handle, prec, L.QMC_RICHTMYER if qmc_type == "Richtmyer" else L.QMC_SOBOL,
                                        C.byref(co), L.ptr(eng, C.c_int32), L.ptr(items, C.c_int32)), ctx.handle)
    return eng, items


def batch_tuning(precision: int, qmc_type="Sobol", *, device: int = 0, context: Optional[Context] = None):
    """The batch engine table in use: -> (engine, item_dims, tuned)."""
    ctx = get_context(device) if context is None else context
    qmc_type = str(qmc_type).lstrip(":")
    eng = np.zeros(513, dtype=np.int32)
    items = np.zeros(513, dtype=np.int32)
    tuned = C.c_int()
    L.check(L.lib().dbgz_batch_tuning(ctx.handle, int(precision),
                                      L.QMC_RICHTMYER if qmc_type == "Richtmyer" else L.QMC_SOBOL,
                                      L.ptr(eng, C.c_int32), L.ptr(items, C.c_int32), C.byref(tuned)), ctx.handle)
    return eng, items, bool(tuned.value)


# ---- primitives -------------------------------------------------------------
def cholesky_genz(M, a, b, block_size=2**7, block_size2=2**9, block_size3=2**10,
                  block_size4=2**11, *, device=0) -> CholeskyGenz:
    """cholesky_genz!(copy(M), copy(a), copy(b), ...) on the GPU (src/cholesky.jl:445)."""
    ctx = get_context(device)
    Mf = np.array(M, dtype=np.float64, order="F", copy=True)
    n = Mf.shape[0]
    a, b = _f64(a).copy(), _f64(b).copy()
    perm = np.zeros(n, dtype=np.int64)
    sv = np.zeros(n)
    rank = C.c_int64()
    L.check(L.lib().dbgz_cholesky_genz(ctx.handle, n, L.ptr(Mf), L.ptr(a), L.ptr(b), block_size,
                                       block_size2, block_size3, block_size4,
                                       L.ptr(perm, C.c_int64), L.ptr(sv), C.byref(rank)), ctx.handle)
    return CholeskyGenz(Mf, perm, rank.value, a, b, block_size, "genz", sv)


def cholesky_classic(M, a, b, block_size=2**7, block_size2=2**9, block_size3=2**10,
                     block_size4=2**11, *, device=0) -> CholeskyGenz:
    """cholesky_classic!(copy(M), copy(a), copy(b), ...) on the GPU (src/cholesky.jl:144)."""
    ctx = get_context(device)
    Mf = np.array(M, dtype=np.float64, order="F", copy=True)
    n = Mf.shape[0]
    a, b = _f64(a).copy(), _f64(b).copy()
    sv = np.zeros(n)
    L.check(L.lib().dbgz_cholesky_classic(ctx.handle, n, L.ptr(Mf), L.ptr(a), L.ptr(b), block_size,
                                          block_size2, block_size3, block_size4, L.ptr(sv)),
            ctx.handle)
    return CholeskyGenz(Mf, np.arange(n), n, a, b, block_size, "none", sv)


def cholesky_rowmax(M, a, b, block_size=2**7, block_size2=2**9, block_size3=2**10,
                    block_size4=2**11, *, device=0) -> CholeskyGenz:
    """cholesky_rowmax!(copy(M), copy(a), copy(b), ...) on the GPU
    (src/cholesky.jl:244-432): diagonal pivoting; a and b come back scaled
    but in the original order, as the reference leaves them."""
    ctx = get_context(device)
    Mf = np.array(M, dtype=np.float64, order="F", copy=True)
    n = Mf.shape[0]
    a, b = _f64(a).copy(), _f64(b).copy()
    perm = np.zeros(n, dtype=np.int64)
    sv = np.zeros(n)
    rank = C.c_int64()
    L.check(L.lib().dbgz_cholesky_rowmax(ctx.handle, n, L.ptr(Mf), L.ptr(a), L.ptr(b), block_size,
                                         block_size2, block_size3, block_size4,
                                         L.ptr(perm, C.c_int64), L.ptr(sv), C.byref(rank)), ctx.handle)
    return CholeskyGenz(Mf, perm, rank.value, a, b, block_size, "row_max", sv)


def adapt_low_rank(M, a, b, rank: int, perm, eps1: float, *, device=0):
    """adapt_low_rank!(M, a, b, rank, perm, eps1) (src/cholesky.jl:24-123) on
    copies -> (M, a, b, perm, k_js, k_0): perm holds 0-based indices, k_js the
    blocks' 1-based end positions (as the reference returns them)."""
    ctx = get_context(device)
    Mf = np.array(M, dtype=np.float64, order="F", copy=True)
    nr, n = Mf.shape
    a, b = _f64(a).copy(), _f64(b).copy()
    pm = np.array(perm, dtype=np.int64, copy=True)
    k_js = np.zeros(max(int(rank), 1), dtype=np.int64)
    k0 = C.c_int64()
    L.check(L.lib().dbgz_adapt_low_rank(ctx.handle, nr, n, L.ptr(Mf), L.ptr(a), L.ptr(b), int(rank),
                                        L.ptr(pm, C.c_int64), float(eps1), L.ptr(k_js, C.c_int64),
                                        C.byref(k0)), ctx.handle)
    return Mf, a, b, pm, k_js[:int(rank)], int(k0.value)


def get_sqrt_primes(n: int) -> np.ndarray:
    q = np.zeros(n)
    L.check(L.lib().dbgz_sqrt_primes(n, L.ptr(q)))
    return q


def richtmyer_mat(m: int, q, n0: int = 0, *, device=0) -> np.ndarray:
    ctx = get_context(device)
    q = _f64(q)
    X = np.zeros((m, q.size), order="F")
    L.check(L.lib().dbgz_richtmyer_mat(ctx.handle, m, q.size, L.ptr(q), n0, L.ptr(X)), ctx.handle)
    return X


def sobol_first_index(m: int, skip0: Optional[int] = None, exact: bool = False) -> int:
    """Index of the first point SobolQMC draws, in the Gray-code order whose
    index 0 is the all-zero point (the index the library's generators take).

    SobolQMC starts from ``skip(SobolSeq(d), skip0)`` with skip0 = 2m - 1
    (src/qmc_generators.jl:57-58).  Sobol.jl 1.5.0's ``skip(s, n)`` (exact =
    false, the default) calls ``next!`` 2^floor(log2(n + 1)) times, and the
    k-th ``next!`` of a fresh sequence returns Gray-code point k (the zero
    point is never returned), so the first point sobol_mat! reads is
    2^floor(log2(2m)) + 1: 2m + 1 when m is a power of two, 16385 for the
    default m = 10^4.  ``exact=True`` restates ``skip(s, n, exact=true)``
    (first point n + 1).  Sobol.jl itself is not part of the reference
    repository; these semantics are its published ones, restated here."""
    n = 2 * int(m) - 1 if skip0 is None else int(skip0)
    if n < 0:
        raise ValueError("skip0 must be non-negative")
    if n == 0:
        return 1
    nskip = n if exact else 1 << ((n + 1).bit_length() - 1)
    return nskip + 1


def sobol_dirnums(dims: int) -> np.ndarray:
    V = np.zeros((dims, 32), dtype=np.uint32)
    L.check(L.lib().dbgz_sobol_dirnums(dims, L.ptr(V, C.c_uint32)))
    return V


def sobol_mat(m: int, V, first: int, *, device=0) -> np.ndarray:
    ctx = get_context(device)
    V = np.ascontiguousarray(V, dtype=np.uint32)
    X = np.zeros((m, V.shape[0]), dtype=np.uint32, order="F")
    L.check(L.lib().dbgz_sobol_mat(ctx.handle, m, V.shape[0], L.ptr(V, C.c_uint32), first,
                                   L.ptr(X, C.c_uint32)), ctx.handle)
    return X

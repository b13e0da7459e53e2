"""ctypes front end of the CPU checker (test infrastructure only).

Loads ``oracle/libgenz_oracle.so`` (built by ``oracle/Makefile``) and exposes
the restated reference functions with numpy arrays.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` import
this module; the product package never does.

All matrices are column-major (Julia layout): a numpy array ``A`` of shape
(n, n) is passed as ``np.asfortranarray(A)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgenz_oracle.so")
_lib = None

RICHTMYER, SOBOL = 0, 1
CDF_ERF, CDF_ERFC = 0, 1


class OrcOpts(C.Structure):
    _fields_ = [
        ("chol_block_size", C.c_int64),
        ("chol_block_size2", C.c_int64),
        ("m", C.c_int64),
        ("block_size_i", C.c_int64),
        ("block_size_i2", C.c_int64),
        ("block_size_j", C.c_int64),
        ("n_reps", C.c_int64),
        ("n_bits", C.c_int64),
        ("max_pts", C.c_int64),
        ("max_abs_err", C.c_double),
    ]


class OrcProblem(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("U", C.POINTER(C.c_double)),
        ("a", C.POINTER(C.c_double)),
        ("b", C.POINTER(C.c_double)),
        ("qmc_type", C.c_int),
        ("q", C.POINTER(C.c_double)),
        ("shifts", C.POINTER(C.c_double)),
        ("V", C.POINTER(C.c_uint32)),
        ("sobol_first", C.c_int64),
        ("ushifts", C.POINTER(C.c_uint64)),
        ("cdf_form", C.c_int),
        ("sparse", C.c_int),
        ("gen_base0", C.c_int64),
        ("logw", C.POINTER(C.c_double)),
    ]


def build() -> str:
    """Compile the checker with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i64, pd, pi64 = C.c_double, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_int64)
        L.orc_det_erf.restype = d
        L.orc_det_erf.argtypes = [d]
        L.orc_det_exp.restype = d
        L.orc_det_exp.argtypes = [d]
        L.orc_erfinv.restype = d
        L.orc_erfinv.argtypes = [d]
        L.orc_cholesky_genz.argtypes = [i64, pd, pd, pd, i64, i64, i64, i64, pi64, pd, pi64]
        L.orc_cholesky_genz_margins.argtypes = [i64, pd, pd, pd, i64, i64, i64, i64, pi64, pd, pi64, pd]
        L.orc_cholesky_classic.argtypes = [i64, pd, pd, pd, i64, i64, i64, i64, pd]
        L.orc_cholesky_rowmax.argtypes = [i64, pd, pd, pd, i64, i64, i64, i64, pi64, pd, pi64]
        L.orc_adapt_low_rank.argtypes = [i64, i64, pd, pd, pd, i64, pi64, d, pi64, pi64]
        L.orc_truncate_U.argtypes = [i64, pd, d]
        L.orc_sqrt_primes.argtypes = [i64, pd]
        L.orc_richtmyer_mat.argtypes = [i64, i64, pd, i64, pd]
        L.orc_sobol_points.argtypes = [i64, C.POINTER(C.c_uint32), i64, i64, C.POINTER(C.c_uint32)]
        L.orc_qmc_pnorm.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcOpts), C.c_int, pd, pd, pi64, pd]
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def det_erf(x: float) -> float:
    return lib().orc_det_erf(float(x))


def det_exp(x: float) -> float:
    return lib().orc_det_exp(float(x))


def erfinv(x: float) -> float:
    return lib().orc_erfinv(float(x))


def cholesky_genz(Sigma, a, b, bs1=64, bs2=512, bs3=1024, bs4=2048, margins=False):
    """cholesky_genz!(copy(Σ), copy(a), copy(b), bs1, bs2) -> dict (src/cholesky.jl:445).
    With margins=True the dict also holds, per pivot step, the gap between the
    winning score and the best other candidate (a diagnostic of near-ties)."""
    n = Sigma.shape[0]
    M = np.array(Sigma, dtype=np.float64, order="F", copy=True)
    a = np.array(a, dtype=np.float64, copy=True)
    b = np.array(b, dtype=np.float64, copy=True)
    perm = np.zeros(n, dtype=np.int64)
    scale = np.zeros(n, dtype=np.float64)
    rank = C.c_int64(0)
    mg = np.full(n, np.nan) if margins else None
    lib().orc_cholesky_genz_margins(n, _pd(M), _pd(a), _pd(b), bs1, bs2, bs3, bs4,
                                    perm.ctypes.data_as(C.POINTER(C.c_int64)), _pd(scale), C.byref(rank),
                                    _pd(mg) if margins else None)
    out = dict(U=M, perm=perm, rank=rank.value, a=a, b=b, scale_vec=scale)
    if margins:
        out["margins"] = mg
    return out


def cholesky_classic(Sigma, a, b, bs1=128, bs2=512, bs3=1024, bs4=2048):
    n = Sigma.shape[0]
    M = np.array(Sigma, dtype=np.float64, order="F", copy=True)
    a = np.array(a, dtype=np.float64, copy=True)
    b = np.array(b, dtype=np.float64, copy=True)
    scale = np.zeros(n, dtype=np.float64)
    lib().orc_cholesky_classic(n, _pd(M), _pd(a), _pd(b), bs1, bs2, bs3, bs4, _pd(scale))
    return dict(U=M, perm=np.arange(n), rank=n, a=a, b=b, scale_vec=scale)


def cholesky_rowmax(Sigma, a, b, bs1=128, bs2=512, bs3=1024, bs4=2048):
    """cholesky_rowmax!(copy(Σ), copy(a), copy(b), bs1, ...) -> dict (src/cholesky.jl:244-432)."""
    n = Sigma.shape[0]
    M = np.array(Sigma, dtype=np.float64, order="F", copy=True)
    a = np.array(a, dtype=np.float64, copy=True)
    b = np.array(b, dtype=np.float64, copy=True)
    perm = np.zeros(n, dtype=np.int64)
    scale = np.zeros(n, dtype=np.float64)
    rank = C.c_int64(0)
    lib().orc_cholesky_rowmax(n, _pd(M), _pd(a), _pd(b), bs1, bs2, bs3, bs4,
                              perm.ctypes.data_as(C.POINTER(C.c_int64)), _pd(scale), C.byref(rank))
    return dict(U=M, perm=perm, rank=rank.value, a=a, b=b, scale_vec=scale)


def adapt_low_rank(M, a, b, rank, perm, eps1):
    """adapt_low_rank!(M, a, b, rank, perm, eps1) on copies -> (M, a, b, perm, k_js, k_0)
    (src/cholesky.jl:24-123); perm 0-based, k_js 1-based block ends."""
    M = np.array(M, dtype=np.float64, order="F", copy=True)
    a = np.array(a, dtype=np.float64, copy=True)
    b = np.array(b, dtype=np.float64, copy=True)
    perm = np.array(perm, dtype=np.int64, copy=True)
    k_js = np.zeros(max(rank, 1), dtype=np.int64)
    k0 = C.c_int64(0)
    lib().orc_adapt_low_rank(M.shape[0], M.shape[1], _pd(M), _pd(a), _pd(b), rank,
                             perm.ctypes.data_as(C.POINTER(C.c_int64)), float(eps1),
                             k_js.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(k0))
    return M, a, b, perm, k_js[:rank], k0.value


def truncate_U(U, eps_T=np.finfo(np.float64).eps):
    U = np.array(U, dtype=np.float64, order="F", copy=True)
    lib().orc_truncate_U(U.shape[0], _pd(U), float(eps_T))
    return U


def sqrt_primes(n):
    q = np.zeros(n, dtype=np.float64)
    lib().orc_sqrt_primes(n, _pd(q))
    return q


def richtmyer_mat(m, q, n0=0):
    q = np.ascontiguousarray(q, dtype=np.float64)
    X = np.zeros((m, q.size), dtype=np.float64, order="F")
    lib().orc_richtmyer_mat(m, q.size, _pd(q), n0, _pd(X))
    return X


def sobol_points(V, first, m):
    V = np.ascontiguousarray(V, dtype=np.uint32)
    dims = V.shape[0]
    X = np.zeros((m, dims), dtype=np.uint32, order="F")
    lib().orc_sobol_points(dims, V.ctypes.data_as(C.POINTER(C.c_uint32)), first, m,
                           X.ctypes.data_as(C.POINTER(C.c_uint32)))
    return X


def qmc_pnorm(U, a, b, *, m, n_reps, qmc_type=RICHTMYER, shifts=None, q=None, V=None,
              sobol_first=0, ushifts=None, cdf_form=CDF_ERF, sparse=False,
              block_size_i=64, block_size_i2=32, block_size_j=64, n_bits=32,
              max_pts=None, max_abs_err=1e-6, threads=0, gen_base0=0, logw=None):
    """qmc_pnorm! on a prepared problem (U, permuted/scaled a, b) -> (P, err, n_pts, reps).
    logw: an (m, n_reps) float64 Fortran-ordered array that receives each
    sample's log-weight (sum of log dc) of the last pass."""
    n = U.shape[0]
    U = np.asfortranarray(U, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    keep = [U, a, b]
    P = OrcProblem()
    P.n = n
    P.U, P.a, P.b = _pd(U), _pd(a), _pd(b)
    P.qmc_type = qmc_type
    P.cdf_form = cdf_form
    P.sparse = 1 if sparse else 0
    P.gen_base0 = int(gen_base0)
    if logw is not None:
        assert logw.shape == (m, n_reps) and logw.dtype == np.float64 and logw.flags.f_contiguous
        P.logw = _pd(logw)
    if qmc_type == RICHTMYER:
        q = sqrt_primes(n - 1) if q is None else np.ascontiguousarray(q, dtype=np.float64)
        sh = np.asfortranarray(shifts, dtype=np.float64)
        assert sh.shape == (n - 1, n_reps)
        keep += [q, sh]
        P.q, P.shifts = _pd(q), _pd(sh)
    else:
        Vv = np.ascontiguousarray(V, dtype=np.uint32)
        us = np.asfortranarray(ushifts, dtype=np.uint64)
        assert us.shape == (n - 1, n_reps) and Vv.shape == (n - 1, 32)
        keep += [Vv, us]
        P.V = Vv.ctypes.data_as(C.POINTER(C.c_uint32))
        P.ushifts = us.ctypes.data_as(C.POINTER(C.c_uint64))
        P.sobol_first = sobol_first
    o = OrcOpts(64, 512, m, block_size_i, block_size_i2, block_size_j, n_reps, n_bits,
                m if max_pts is None else max_pts, max_abs_err)
    res, err, npts = C.c_double(0), C.c_double(0), C.c_int64(0)
    reps = np.zeros(n_reps, dtype=np.float64)
    lib().orc_qmc_pnorm(C.byref(P), C.byref(o), threads, C.byref(res), C.byref(err),
                        C.byref(npts), _pd(reps))
    del keep
    return res.value, err.value, npts.value, reps


# ---- the timed CPU baseline (oracle/genz_cpu_blas.c) ----------------------
class CpuProblem(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("U", C.POINTER(C.c_double)),
        ("a", C.POINTER(C.c_double)),
        ("b", C.POINTER(C.c_double)),
        ("qmc_type", C.c_int),
        ("q", C.POINTER(C.c_double)),
        ("shifts", C.POINTER(C.c_double)),
        ("V", C.POINTER(C.c_uint32)),
        ("sobol_first", C.c_int64),
        ("ushifts", C.POINTER(C.c_uint64)),
        ("n_bits", C.c_int64),
    ]


_cpu = None


def cpu_isa() -> str:
    """'avx512' when the host CPU has AVX-512 (F, DQ, BW, VL), else 'avx2'."""
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return "avx2"
    return "avx512" if all(f" {x}" in flags for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl")) else "avx2"


def openblas_path() -> str:
    """numpy's bundled OpenBLAS (ILP64, symbols with the scipy_ prefix)."""
    import glob
    base = os.path.dirname(os.path.dirname(np.__file__))
    cand = sorted(glob.glob(os.path.join(base, "numpy.libs", "libscipy_openblas64_*.so")))
    if not cand:
        raise RuntimeError("numpy's bundled OpenBLAS (libscipy_openblas64_*.so) not found")
    return cand[0]


def cpu_lib():
    """The vectorised BLAS-3 CPU loop for this CPU, with dgemm bound."""
    global _cpu
    if _cpu is None:
        path = os.path.join(_HERE, f"libgenz_cpu_{cpu_isa()}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.cpu_blas_init.argtypes = [C.c_char_p]
        L.cpu_qmc_pass.argtypes = [C.POINTER(CpuProblem), C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                   C.c_double, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                                   C.POINTER(C.c_double)]
        L.cpu_erfinv.argtypes = [C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        rc = L.cpu_blas_init(openblas_path().encode())
        if rc != 0:
            raise RuntimeError(f"cpu_blas_init failed ({rc})")
        _cpu = L
    return _cpu


def cpu_erfinv(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    cpu_lib().cpu_erfinv(x.size, _pd(x), _pd(y))
    return y


def first_cdf(U, a, b):
    """c_1, dc_1 of qmc_pnorm! (src/qmc.jl:800-809, erf form)."""
    import math
    c2 = math.sqrt(2.0)
    aa = a[0] / (U[0, 0] * c2)
    bb = b[0] / (U[0, 0] * c2)
    return 0.5 * (1 + math.erf(aa)), 0.5 * (math.erf(bb) - math.erf(aa))


def qmc_pass_blas(U, a, b, *, m, n_reps, qmc_type=RICHTMYER, shifts=None, q=None, V=None, sobol_first=0,
                  ushifts=None, n_bits=32, block_size_i=512, block_size_i2=64, block_size_j=64,
                  threads=0, n_pass_base=0):
    """One qmc_loop! pass of the BLAS-3, vectorised CPU restatement (the timed
    baseline); returns the per-shift means (first pass, n_pts0 = 0).  Default
    blocks are the reference's x86/MKL paper settings (block_size_i 2^9,
    block_size_i2 2^6, block_size_j 2^6: scripts/simulations/simulation_comparison.jl:33-34)."""
    n = U.shape[0]
    U = np.asfortranarray(U, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    keep = [U, a, b]
    P = CpuProblem()
    P.n = n
    P.U, P.a, P.b = _pd(U), _pd(a), _pd(b)
    P.qmc_type = qmc_type
    P.n_bits = n_bits
    if qmc_type == RICHTMYER:
        q = sqrt_primes(n - 1) if q is None else np.ascontiguousarray(q, dtype=np.float64)
        sh = np.asfortranarray(shifts, dtype=np.float64)
        assert sh.shape == (n - 1, n_reps)
        keep += [q, sh]
        P.q, P.shifts = _pd(q), _pd(sh)
    else:
        Vv = np.ascontiguousarray(V, dtype=np.uint32)
        us = np.asfortranarray(ushifts, dtype=np.uint64)
        assert us.shape == (n - 1, n_reps) and Vv.shape == (n - 1, 32)
        keep += [Vv, us]
        P.V = Vv.ctypes.data_as(C.POINTER(C.c_uint32))
        P.ushifts = us.ctypes.data_as(C.POINTER(C.c_uint64))
        P.sobol_first = sobol_first
    c1, dc1 = first_cdf(U, a, b)
    reps = np.zeros(n_reps, dtype=np.float64)
    rc = cpu_lib().cpu_qmc_pass(C.byref(P), m, n_reps, 0, n_pass_base, c1, dc1, block_size_i,
                                block_size_i2, block_size_j, threads, _pd(reps))
    if rc != 0:
        raise RuntimeError(f"cpu_qmc_pass failed ({rc})")
    del keep
    return reps

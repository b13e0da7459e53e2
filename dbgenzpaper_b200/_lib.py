"""ctypes binding of libdbgenz.so (the C ABI declared in include/dbgenz.h).

The library is loaded from the package directory.  There is no fallback:
if it is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdbgenz.so")
HEADER = os.path.join(HERE, "..", "include", "dbgenz.h")

# status codes (dbgz_status)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_RANK_DEFICIENT = 2
ERR_NONFINITE_INPUT = 3
ERR_DIMENSION = 4
ERR_OUT_OF_MEMORY = 5
ERR_CUDA = 6
ERR_TIMEOUT = 7
ERR_UNSUPPORTED = 8

QMC_RICHTMYER, QMC_SOBOL = 0, 1
STRUCTURE_DENSE, STRUCTURE_SPARSE = 0, 1
CDF_ERF, CDF_ERFC = 0, 1
PREC_FP64, PREC_FP32_TF32, PREC_FP32_SPLIT_BF16, PREC_FP32_SIMT = 0, 1, 2, 3


class DbgzOpts(C.Structure):
    _fields_ = [
        ("chol_block_size", C.c_int64),
        ("chol_block_size2", C.c_int64),
        ("m", C.c_int64),
        ("block_size_i", C.c_int64),
        ("block_size_i2", C.c_int64),
        ("block_size_j", C.c_int64),
        ("n_blocks", C.c_int64),
        ("n_reps", C.c_int64),
        ("n_bits", C.c_int64),
        ("max_pts", C.c_int64),
        ("max_abs_err", C.c_double),
    ]


class DbgzProfile(C.Structure):
    _fields_ = [
        ("pnorm_ms", C.c_double),
        ("loop_ms", C.c_double),
        ("finalize_ms", C.c_double),
        ("loop_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("prepare_ms", C.c_double),
        ("prepare_launches", C.c_int64),
        ("sigma_adjoint_ms", C.c_double),
        ("grad_state_bytes", C.c_int64),
        ("grad_chunks", C.c_int64),
    ]


class DbgzError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib = None

_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)
_pu32 = C.POINTER(C.c_uint32)
_pu64 = C.POINTER(C.c_uint64)
_vp = C.c_void_p

# name -> (restype, argtypes); kept in step with include/dbgenz.h
SIGNATURES = {
    "dbgz_abi_version": (C.c_int, []),
    "dbgz_default_opts": (None, [C.POINTER(DbgzOpts)]),
    "dbgz_status_string": (C.c_char_p, [C.c_int]),
    "dbgz_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "dbgz_destroy": (C.c_int, [_vp]),
    "dbgz_release_cached": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "dbgz_set_state_budget": (C.c_int, [_vp, C.c_uint64]),
    "dbgz_last_error": (C.c_char_p, [_vp]),
    "dbgz_set_profiling": (C.c_int, [_vp, C.c_int]),
    "dbgz_get_profile": (C.c_int, [_vp, C.POINTER(DbgzProfile)]),
    "dbgz_prepare": (C.c_int, [_vp, C.c_int64, _pd, _pd, _pd, C.POINTER(DbgzOpts), C.c_int,
                               C.c_int, C.c_int, _pd, _pu64, _pu32, C.c_int64, C.POINTER(_vp)]),
    "dbgz_problem_free": (C.c_int, [_vp]),
    "dbgz_problem_set_cdf_form": (C.c_int, [_vp, C.c_int]),
    "dbgz_problem_truncate_band": (C.c_int, [_vp, C.c_int64]),
    "dbgz_problem_factor": (C.c_int, [_vp, _pd, _pi64, _pd, _pd, _pd, _pi64]),
    "dbgz_pnorm": (C.c_int, [_vp, C.c_int, _pd, _pd, _pi64, _pd]),
    "dbgz_pnorm_logw": (C.c_int, [_vp, C.c_int, _pd, _pd]),
    "dbgz_set_grad_checkpoints": (C.c_int, [_vp, C.c_int64]),
    "dbgz_pnorm_graph": (C.c_int, [_vp, C.c_int, _pd, _pd, _pi64, _pd]),
    "dbgz_pnorm_grad": (C.c_int, [_vp, C.c_int, _pd, _pd, _pi64, _pd, _pd, _pd]),
    "dbgz_problem_sigma_adjoint": (C.c_int, [_vp, _pd, _pd, _pd, _pd]),
    "dbgz_pnorm_grad_sigma": (C.c_int, [_vp, C.c_int, _pd, _pd, _pi64, _pd, _pd, _pd]),
    "dbgz_pnorm_batch": (C.c_int, [_vp, C.c_int64, _pi64, _pd, _pd, _pd, C.POINTER(DbgzOpts), C.c_int, C.c_int,
                                   _pd, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.c_int64, _pd, _pd,
                                   _pi64]),
    "dbgz_batch_plan_create": (C.c_int, [_vp, C.c_int64, _pi64, C.POINTER(DbgzOpts), C.c_int, C.c_int, _pu32,
                                         C.c_int64, C.POINTER(_vp)]),
    "dbgz_batch_plan_buffers": (C.c_int, [_vp, C.POINTER(_pd), C.POINTER(_pd), C.POINTER(_pd), C.POINTER(_vp)]),
    "dbgz_batch_plan_run": (C.c_int, [_vp, _pd, _pd, _pi64]),
    "dbgz_batch_plan_info": (C.c_int, [_vp, _pi64, _pi64, _pi64, _pi64]),
    "dbgz_batch_plan_destroy": (C.c_int, [_vp]),
    "dbgz_batch_autotune": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(DbgzOpts), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32)]),
    "dbgz_batch_tuning": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int)]),
    "dbgz_pnorm_pass_noalloc": (C.c_int, [C.c_int64, _vp, _vp, _vp, _vp, _vp, C.c_int64,
                                          C.c_int64, C.c_int64, _vp, _vp]),
    "dbgz_cholesky_genz": (C.c_int, [_vp, C.c_int64, _pd, _pd, _pd, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_int64, _pi64, _pd, _pi64]),
    "dbgz_cholesky_rowmax": (C.c_int, [_vp, C.c_int64, _pd, _pd, _pd, C.c_int64, C.c_int64, C.c_int64,
                                       C.c_int64, _pi64, _pd, _pi64]),
    "dbgz_adapt_low_rank": (C.c_int, [_vp, C.c_int64, C.c_int64, _pd, _pd, _pd, C.c_int64, _pi64, C.c_double,
                                      _pi64, _pi64]),
    "dbgz_cholesky_classic": (C.c_int, [_vp, C.c_int64, _pd, _pd, _pd, C.c_int64, C.c_int64,
                                        C.c_int64, C.c_int64, _pd]),
    "dbgz_sqrt_primes": (C.c_int, [C.c_int64, _pd]),
    "dbgz_richtmyer_mat": (C.c_int, [_vp, C.c_int64, C.c_int64, _pd, C.c_int64, _pd]),
    "dbgz_sobol_mat": (C.c_int, [_vp, C.c_int64, C.c_int64, _pu32, C.c_int64, _pu32]),
    "dbgz_sobol_dirnums": (C.c_int, [C.c_int64, _pu32]),
}


def header_symbols() -> list[str]:
    """Every function name declared in include/dbgenz.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dbgz_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Load libdbgenz.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; run `python -m dbgenzpaper_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a, ctype=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def check(status: int, ctx=None) -> None:
    if status != OK:
        L = lib()
        msg = L.dbgz_status_string(status).decode()
        if ctx is not None:
            detail = L.dbgz_last_error(ctx)
            if detail:
                msg = f"{msg}: {detail.decode()}"
        raise DbgzError(status, msg)

"""The C ABI library without a GPU: it loads, exports every symbol
include/dbgenz.h declares, validates arguments, and its host-only helpers
agree with the checker.  No device compute is called here."""
import ctypes as C

import numpy as np
import pytest

from dbgenzpaper_b200 import _lib as L


@pytest.fixture(scope="module")
def lib(dbgz):
    return L.lib()


def test_exports_every_declared_symbol(lib):
    syms = L.header_symbols()
    assert len(syms) >= 17
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(L.SIGNATURES), "ctypes signatures out of step with the header"
    assert lib.dbgz_abi_version() == 1


def test_default_opts_match_reference(lib, dbgz):
    o = L.DbgzOpts()
    lib.dbgz_default_opts(C.byref(o))
    ref = dbgz.QMC_opts()  # src/qmc.jl:111-125 defaults
    for f in ("chol_block_size", "chol_block_size2", "m", "block_size_i", "block_size_i2",
              "block_size_j", "n_reps", "n_bits", "max_pts"):
        assert getattr(o, f) == getattr(ref, f), f
    assert o.max_abs_err == ref.max_abs_err == 1e-6


def test_status_strings(lib):
    assert lib.dbgz_status_string(0) == b"ok"
    assert b"full-rank" in lib.dbgz_status_string(L.ERR_RANK_DEFICIENT)
    assert lib.dbgz_status_string(99) == b"unknown status"


def test_null_arguments_rejected_without_device(lib):
    out = C.c_void_p()
    assert lib.dbgz_create(0, None) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_prepare(None, 3, None, None, None, None, 0, 0, 0, None, None, None, 0,
                            C.byref(out)) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_prepare(None, 3, None, None, None, None, 0, 0, 0, None, None, None, 0,
                            None) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_pnorm(None, 0, None, None, None, None) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_problem_free(None) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_problem_set_cdf_form(None, 0) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_destroy(None) == L.ERR_INVALID_ARGUMENT
    assert lib.dbgz_sqrt_primes(-1, None) == L.ERR_INVALID_ARGUMENT


def test_no_cpu_fallback_without_device(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert lib.dbgz_create(0, C.byref(h)) == L.ERR_CUDA
    assert not h.value


def test_sqrt_primes_match_checker(lib, oracle):
    n = 2000
    q = np.zeros(n)
    assert lib.dbgz_sqrt_primes(n, q.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert np.array_equal(q, oracle.sqrt_primes(n))


def test_sobol_direction_numbers(lib):
    dims = 10_000  # the d = 10^4 banded configuration needs 9999
    V = np.zeros((dims, 32), dtype=np.uint32)
    assert lib.dbgz_sobol_dirnums(dims, V.ctypes.data_as(C.POINTER(C.c_uint32))) == 0
    k = np.arange(32, dtype=np.uint64)
    m = V.astype(np.uint64) >> (31 - k)[None, :]
    assert np.all(m & 1 == 1)                     # every m_k odd
    assert np.all(m < (2 * 2 ** k)[None, :])       # m_k < 2^k
    assert np.all(V[:, 0] == 2**31)
    assert len({tuple(r) for r in V[:, :20]}) == dims  # distinct dimensions


def test_python_mirror_options(dbgz):
    o = dbgz.QMC_opts(np.float32, m=32, n_reps=2)
    assert o.T is np.float32 and o.m == 32 and o.n_reps == 2 and o.chol_block_size == 64
    with pytest.raises(TypeError):
        dbgz.QMC_opts(np.int32)

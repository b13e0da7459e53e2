"""The FP64 dense kernels of the gradient path (dense64.cuh: the Cholesky
adjoint's products and triangular inverse, the FP64 factor-gradient GEMM)
against numpy (needs a B200), through tests/csrc/dense64_unit.cu: every
operand transposition, the triangular k ranges, the three output rules,
split-K with accumulation, sizes that are not multiples of the 64 x 64 tile."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "dense64_unit.cu")
HDR = os.path.join(HERE, "..", "dbgenzpaper_b200", "csrc", "dense64.cuh")
LIB = os.path.join(HERE, "csrc", "libdense64_unit.so")
FULL, LOWER_PHI, STRICT_UPPER = 0, 1, 2


@pytest.fixture(scope="module")
def lib():
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HDR))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
                        "-Xcompiler", "-fPIC", "-o", LIB, SRC], check=True)
    L = C.CDLL(LIB)
    pd = C.POINTER(C.c_double)
    L.dense64_gemm.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, pd, C.c_int64, pd, C.c_int64, pd,
                               C.c_int64] + [C.c_int] * 7
    L.dense64_trinv.argtypes = [C.c_int64, pd, pd]
    return L


def _p(x):
    return x.ctypes.data_as(C.POINTER(C.c_double))


def _gemm(lib, ta, tb, A, B, C0, **kw):
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    Cm = np.asfortranarray(C0.copy())
    m, n = Cm.shape
    k = A.shape[0] if ta else A.shape[1]
    rc = lib.dense64_gemm(int(ta), int(tb), m, n, k, _p(A), A.shape[0], _p(B), B.shape[0], _p(Cm), m,
                          kw.get("kmin_row", 0), kw.get("kmin_col", 0), kw.get("kmax_row", 0),
                          kw.get("kmax_col", 0), kw.get("out", FULL), kw.get("accumulate", 0), kw.get("splits", 1))
    assert rc == 0
    return Cm


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(64, 64, 64), (100, 37, 250), (1, 130, 17), (129, 65, 1000)])
def test_gemm_plain(lib, ta, tb, m, n, k):
    rng = np.random.default_rng(m * 1000 + n + k)
    A = rng.standard_normal((k, m) if ta else (m, k))
    B = rng.standard_normal((n, k) if tb else (k, n))
    ref = (A.T if ta else A) @ (B.T if tb else B)
    got = _gemm(lib, ta, tb, A, B, np.zeros((m, n)))
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-12 * np.sqrt(k))


def test_gemm_triangles_and_rules(lib):
    rng = np.random.default_rng(3)
    d = 203
    U = np.triu(rng.standard_normal((d, d)))
    Lb = np.tril(rng.standard_normal((d, d)))
    # Phi(U Lb): lower triangle, halved diagonal, upper zero; k >= max(i, j)
    ref = U @ Lb
    ref = np.tril(ref, -1) + 0.5 * np.diag(np.diag(ref))
    got = _gemm(lib, 0, 0, U, Lb, np.zeros((d, d)), kmin_row=1, kmin_col=1, out=LOWER_PHI)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-11)
    # U' U over k <= min(i, j)
    got = _gemm(lib, 1, 0, U, U, np.zeros((d, d)), kmax_row=1, kmax_col=1)
    np.testing.assert_allclose(got, U.T @ U, rtol=1e-13, atol=1e-11)
    # X V' with V upper: k >= j
    X = rng.standard_normal((d, d))
    got = _gemm(lib, 0, 1, X, U, np.zeros((d, d)), kmin_col=1)
    np.testing.assert_allclose(got, X @ U.T, rtol=1e-13, atol=1e-11)


@pytest.mark.parametrize("splits", [1, 3, 8])
def test_gemm_split_k_strict_upper_accumulate(lib, splits):
    # the factor-gradient shape: C[l, t] += sum_n Y[n, l] S[n, t] for l < t
    rng = np.random.default_rng(splits)
    N, d = 5000, 150
    Y = rng.standard_normal((N, d))
    S = rng.standard_normal((N, d))
    C0 = rng.standard_normal((d, d))
    got = _gemm(lib, 1, 0, Y, S, C0, out=STRICT_UPPER, accumulate=1, splits=splits)
    ref = C0.copy()
    iu = np.triu_indices(d, 1)
    ref[iu] += (Y.T @ S)[iu]
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("d", [1, 5, 64, 333, 1000, 1500, 2500])
def test_trinv(lib, d):
    rng = np.random.default_rng(d)
    A = rng.standard_normal((d, d + 5))
    R = np.linalg.cholesky(A @ A.T + d * np.eye(d)).T  # upper, well conditioned
    Uj = np.asfortranarray(R + np.tril(rng.standard_normal((d, d)), -1))  # lower triangle junk is ignored
    X = np.zeros((d, d), order="F")
    assert lib.dense64_trinv(d, _p(Uj), _p(X)) == 0
    np.testing.assert_allclose(X, np.linalg.inv(R), rtol=1e-12, atol=1e-13)
    assert np.all(np.tril(X, -1) == 0)

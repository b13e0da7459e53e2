"""tcgen05 / TMA conventions in isolation (needs a B200): one 128 x N x 32
product per case through tests/csrc/umma_unit.cu, in the split-BF16 and TF32
forms, with the swizzled layouts, B row offsets and TMEM column offsets the
tensor-core loop uses.  Compared with the same split products in float64."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "umma_unit.cu")
LIB = os.path.join(HERE, "csrc", "libumma_unit.so")


def build_unit():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-std=c++17", "-shared",
               "-Xcompiler", "-fPIC", "-o", LIB, SRC]
        subprocess.run(cmd, check=True)
    L = C.CDLL(LIB)
    pf = C.POINTER(C.c_float)
    L.umma_unit.argtypes = [C.c_int, C.c_int, C.c_int, pf, pf, pf, C.c_int, C.c_int]
    return L


def bf16_round(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def tf32_round(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x1000) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


@pytest.fixture(scope="module")
def unit():
    return build_unit()


CASES = [(N, br, dc) for N in (32, 64, 96, 224, 256) for br, dc in ((0, 0), (32, 32), (0, 64))
         if dc + N <= 256]


@pytest.mark.parametrize("mode", [2, 1])
@pytest.mark.parametrize("N,b_row,d_col", CASES)
def test_umma_product(unit, mode, N, b_row, d_col):
    rng = np.random.default_rng(N * 7 + b_row + d_col + mode)
    rows = b_row + ((N + 63) // 64) * 64
    A = rng.standard_normal((128, 32)).astype(np.float32) * 2.0
    B = (rng.standard_normal((rows, 32)) * 0.05).astype(np.float32)
    D = np.full((128, N), np.nan, dtype=np.float32)
    pf = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    rc = unit.umma_unit(mode, N, rows, pf(A), pf(B), pf(D), b_row, d_col)
    assert rc == 0
    Bs = B[b_row:b_row + N].astype(np.float64)
    if mode == 2:
        Ah = bf16_round(A).astype(np.float64)
        Al = bf16_round(A - bf16_round(A)).astype(np.float64)
        Bh = bf16_round(B[b_row:b_row + N]).astype(np.float64)
        Bl = bf16_round(B[b_row:b_row + N] - bf16_round(B[b_row:b_row + N])).astype(np.float64)
        ref = Ah @ Bh.T + Ah @ Bl.T + Al @ Bh.T
    else:
        ref = tf32_round(A).astype(np.float64) @ tf32_round(B[b_row:b_row + N]).astype(np.float64).T
    scale = np.abs(A).astype(np.float64) @ np.abs(Bs).T + 1e-30
    assert np.all(np.isfinite(D))
    assert np.max(np.abs(D - ref) / scale) < 2e-6
    # and the split product reproduces the exact FP32 product to ~2^-16
    if mode == 2:
        exact = A.astype(np.float64) @ Bs.T
        assert np.max(np.abs(D - exact) / scale) < 5e-5

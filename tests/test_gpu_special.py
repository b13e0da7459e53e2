"""The FP32 tail mass and inverse normal of the mixed-precision step
(csrc/normal32.cuh) against erfc and the normal quantile in float64 on dense
grids of FP32 inputs (needs a B200)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
from scipy.special import erfc, ndtri

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "special_unit.cu")
HDR = os.path.join(HERE, "..", "dbgenzpaper_b200", "csrc", "normal32.cuh")
LIB = os.path.join(HERE, "csrc", "libspecial_unit.so")


def _lib():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
                        "-Xcompiler", "-fPIC", "-o", LIB, SRC], check=True)
    L = C.CDLL(LIB)
    pf = C.POINTER(C.c_float)
    L.tail_mass_eval.argtypes = [pf, pf, C.c_int]
    L.phi_inv_eval.argtypes = [pf, pf, C.c_int]
    return L


def test_tail_mass_relative_error():
    L = _lib()
    x = np.linspace(0.0, 9.0, 900001).astype(np.float32)
    out = np.zeros_like(x)
    pf = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    assert L.tail_mass_eval(pf(x), pf(out), x.size) == 0
    ref = 0.5 * erfc(x.astype(np.float64))
    rel = np.abs(out.astype(np.float64) / ref - 1.0)
    near = x <= 4.5
    assert rel[near].max() < 3e-6, rel[near].max()
    assert rel.max() < 1.5e-5, rel.max()
    assert out[0] == pytest.approx(0.5, rel=1e-6) and np.all(np.diff(out) <= 0)


def test_phi_inv_lower_relative_error():
    L = _lib()
    p = np.exp(np.linspace(np.log(2.3e-16), np.log(0.5), 2000001)).astype(np.float32)
    p = np.unique(p[(p > 0) & (p <= 0.5)])
    out = np.zeros_like(p)
    pf = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    assert L.phi_inv_eval(pf(p), pf(out), p.size) == 0
    ref = ndtri(p.astype(np.float64))
    far = p < 0.45  # away from the zero of Phi^-1 at 1/2
    rel = np.abs(out[far].astype(np.float64) / ref[far] - 1.0)
    assert rel.max() < 5e-7, rel.max()
    assert np.all(np.abs(out[~far] - ref[~far]) < 2e-8 + 5e-7 * np.abs(ref[~far]))
    assert out[-1] == 0.0

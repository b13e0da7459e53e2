"""The adaptive loop of qmc_pnorm! driven on the device (dbgz_pnorm_graph:
one CUDA graph with a conditional while node) against the host-driven loop
(dbgz_pnorm): the same bits, the same number of points, the same generator
state across calls (needs a B200)."""
import numpy as np
import pytest

from dbgenzpaper_b200 import _lib as L
from dbgenzpaper_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _case(d, seed):
    rng = np.random.default_rng(seed)
    S = W.rand_spd(d, 1.0, rng)
    a = rng.uniform(-2.0, -0.2, d) * np.sqrt(np.diag(S))
    b = rng.uniform(0.2, 2.0, d) * np.sqrt(np.diag(S))
    return S, a, b, rng


def _pair(D, S, a, b, opts, qmc, rng, cls=None):
    cls = cls or D.QMCData
    R = opts.n_reps
    if qmc == "Richtmyer":
        kw = dict(qmc_type=qmc, shifts=rng.random((len(a) - 1, R)))
    else:
        kw = dict(qmc_type=qmc, ushifts=rng.integers(0, 2**63, size=(len(a) - 1, R), dtype=np.uint64))
    return cls(S, a, b, opts, **kw), cls(S, a, b, opts, **kw)


@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol"])
@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32_SIMT, L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
def test_graph_driver_equals_host_loop(dbgz, qmc, prec):
    D = dbgz
    S, a, b, rng = _case(40, 7)
    opts = D.QMC_opts(m=640, n_reps=6, max_pts=640 * 7, max_abs_err=0.0)  # runs to max_pts: 7 passes
    Qh, Qg = _pair(D, S, a, b, opts, qmc, rng)
    try:
        for _ in range(2):  # the second call continues the point sequence
            rh = D.qmc_pnorm(Qh, precision=prec, return_reps=True)
            rg = D.qmc_pnorm(Qg, precision=prec, return_reps=True, driver="graph")
            assert rh[2] == rg[2] == 640 * 7
            assert rh[0] == rg[0] and rh[1] == rg[1], (rh[:2], rg[:2])
            assert np.array_equal(rh[3], rg[3])
    finally:
        Qh.close()
        Qg.close()


def test_graph_driver_early_stop_and_tolerance(dbgz):
    D = dbgz
    S, a, b, rng = _case(12, 9)
    for tol in (1e-1, 2e-4, 0.0):
        opts = D.QMC_opts(m=1000, n_reps=8, max_pts=20000, max_abs_err=tol)
        Qh, Qg = _pair(D, S, a, b, opts, "Richtmyer", np.random.default_rng(3))
        try:
            rh = D.qmc_pnorm(Qh, precision=L.PREC_FP64)
            rg = D.qmc_pnorm(Qg, precision=L.PREC_FP64, driver="graph")
            assert rh == rg
            if tol == 1e-1:
                assert rg[2] == 1000  # the first pass already meets the tolerance
            if tol == 0.0:
                assert rg[2] == 20000
        finally:
            Qh.close()
            Qg.close()


def test_graph_driver_sparse_and_erfc_form(dbgz):
    D = dbgz
    S, a, b, rng = _case(60, 11)
    opts = D.QMC_opts(m=512, n_reps=4, max_pts=512 * 3, max_abs_err=0.0)
    Qh, Qg = _pair(D, S, a, b, opts, "Sobol", rng, cls=D.QMCDataSparse)
    try:
        for prec in (L.PREC_FP64, L.PREC_FP32_SIMT):
            assert D.qmc_pnorm(Qh, precision=prec) == D.qmc_pnorm(Qg, precision=prec, driver="graph")
    finally:
        Qh.close()
        Qg.close()
    Qh, Qg = _pair(D, S, a, b, opts, "Richtmyer", rng)
    try:
        # erfc form (the graph is rebuilt when the CDF form changes), then erf again
        rh = D.qmc_pnorm(D.QMCData_Distributions(Qh), precision=L.PREC_FP64)
        rg = D.qmc_pnorm(D.QMCData_Distributions(Qg), precision=L.PREC_FP64, driver="graph")
        assert rh == rg
        assert D.qmc_pnorm(Qh, precision=L.PREC_FP64) == D.qmc_pnorm(Qg, precision=L.PREC_FP64, driver="graph")
    finally:
        Qh.close()
        Qg.close()


def test_graph_driver_after_gradient_call(dbgz):
    # a gradient call resizes the problem's buffers: the cached graph must be
    # rebuilt, not replayed on stale addresses
    D = dbgz
    S, a, b, rng = _case(30, 13)
    opts = D.QMC_opts(m=2048, n_reps=4, max_pts=2048 * 2, max_abs_err=0.0)
    Qh, Qg = _pair(D, S, a, b, opts, "Richtmyer", rng)
    try:
        assert D.qmc_pnorm(Qh, precision=L.PREC_FP32_SPLIT_BF16) == \
            D.qmc_pnorm(Qg, precision=L.PREC_FP32_SPLIT_BF16, driver="graph")
        D.qmc_pnorm_grad(Qh, precision=L.PREC_FP32_SPLIT_BF16)
        D.qmc_pnorm_grad(Qg, precision=L.PREC_FP32_SPLIT_BF16)
        assert D.qmc_pnorm(Qh, precision=L.PREC_FP32_SPLIT_BF16) == \
            D.qmc_pnorm(Qg, precision=L.PREC_FP32_SPLIT_BF16, driver="graph")
    finally:
        Qh.close()
        Qg.close()

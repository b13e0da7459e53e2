"""CUDA path against the CPU checker at the benchmark configurations' own
shapes (needs a B200), with fewer points so the checker finishes in seconds.

- d = 1000 factor-model covariance (B 1000 x 20, the metric's workload):
  the factorisation bit for bit at its own bounds and at the reference's
  bound design; FP64 per-shift means within 1e-12 of the checker and the
  mixed-precision modes within their tolerances of the checker (not of the
  GPU's own FP64 path) where P is O(0.1).
- The same covariance at its own bounds (1000 thresholds at marginal
  probabilities 1e-3..1e-1), where P underflows to 0 in FP64: per-sample
  log-weights (dbgz_pnorm_logw) against the checker's, and the
  mixed-precision estimate against FP64 in log space.
- d = 500 random correlation, finite bounds, Sobol points (the precision
  comparison configuration): FP64 within 1e-12 of the checker, the
  mixed-precision modes within their tolerances of the checker.
"""
import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L

pytestmark = pytest.mark.gpu

MIXED = [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32, L.PREC_FP32_SIMT]
# |P - P_checker| <= atol + rtol P, as in the other parity tests
TOL = {L.PREC_FP32_SPLIT_BF16: (5e-6, 2e-5), L.PREC_FP32_TF32: (1e-4, 2e-3), L.PREC_FP32_SIMT: (2e-6, 1e-5)}


@pytest.fixture(scope="module")
def D(dbgz):
    dbgz.get_context(0)
    return dbgz


def _opts(D, m, R):
    return D.QMC_opts(m=m, n_reps=R, max_pts=m, max_abs_err=0.0)


@pytest.mark.parametrize("quarter", [False, True])
def test_d1000_factor_bitexact(D, oracle, quarter):
    w = (W.c3_quarter if quarter else W.c3)(d=1000, m=256, n_reps=2)
    G = D.cholesky_genz(w.Sigma, w.a, w.b, 64, 512)  # QMC_opts' chol_block_size(2)
    F = oracle.cholesky_genz(w.Sigma, w.a, w.b, 64, 512)
    assert G.rank == F["rank"] == 1000
    assert np.array_equal(G.perm, F["perm"])
    assert np.array_equal(G.U, F["U"])
    assert np.array_equal(G.a, F["a"]) and np.array_equal(G.b, F["b"])


def test_d1000_quarter_bounds_vs_checker(D, oracle):
    m, R = 512, 2
    w = W.c3_quarter(d=1000, m=m, n_reps=R)
    Q = D.QMCData(w.Sigma, w.a, w.b, _opts(D, m, R), shifts=w.shifts)
    try:
        out = {pr: D.qmc_pnorm(Q, precision=pr, return_reps=True) for pr in [L.PREC_FP64] + MIXED}
        F = Q.C
        Pc, ec, nc, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=m, n_reps=R, shifts=w.shifts, max_pts=m,
                                          max_abs_err=0.0)
    finally:
        Q.close()
    np.testing.assert_allclose(out[L.PREC_FP64][3], rc, rtol=1e-12, atol=0)
    assert 0.05 < Pc < 0.95
    for pr in MIXED:
        at, rt = TOL[pr]
        np.testing.assert_allclose(out[pr][3], rc, rtol=0, atol=at + rt * abs(Pc), err_msg=f"precision {pr}")


def test_d1000_own_bounds_logweights(D, oracle):
    """At the metric's own bounds the erf form of the CDF (src/qmc.jl:405-429)
    rounds erf(x) to -1 below x = -5.9 and gives dc = 0 exactly somewhere in
    (nearly) every sample, so P is 0 in FP64 structurally, not only by
    underflow.  The erfc form (QMCData_Distributions, src/qmc.jl:587-593)
    keeps those tails: its log-weights are finite and are compared with the
    checker's, and the mixed-precision modes (whose tail masses are of the
    erfc form) with them in log space."""
    m, R = 256, 2
    w = W.c3(d=1000, m=m, n_reps=R)
    Q = D.QMCData(w.Sigma, w.a, w.b, _opts(D, m, R), shifts=w.shifts)
    Qc = D.QMCData(w.Sigma, w.a, w.b, _opts(D, m, R), shifts=w.shifts, cdf_form=L.CDF_ERFC)
    try:
        lw_erf = D.qmc_pnorm_logw(Q, precision=L.PREC_FP64)[0]
        lw = {pr: D.qmc_pnorm_logw(Qc, precision=pr)[0] for pr in [L.PREC_FP64] + MIXED}
        P64 = D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]
        F = Q.C
        lwc = np.zeros((m, R), order="F")
        oracle.qmc_pnorm(F.U, F.a, F.b, m=m, n_reps=R, shifts=w.shifts, max_pts=m, max_abs_err=0.0, logw=lwc,
                         cdf_form=oracle.CDF_ERFC)
        lwc_erf = np.zeros((m, R), order="F")
        oracle.qmc_pnorm(F.U, F.a, F.b, m=m, n_reps=R, shifts=w.shifts, max_pts=m, max_abs_err=0.0, logw=lwc_erf)
    finally:
        Q.close()
        Qc.close()
    assert P64 == 0.0
    # the erf form: the same zero factors as the checker
    assert np.array_equal(np.isneginf(lw_erf), np.isneginf(lwc_erf))
    fin = np.isfinite(lwc_erf)
    np.testing.assert_allclose(lw_erf[fin], lwc_erf[fin], rtol=1e-12, atol=1e-9)
    # the erfc form: finite log-weights (P underflows, they do not)
    assert np.all(np.isfinite(lwc)) and np.all(lwc < -700)
    np.testing.assert_allclose(lw[L.PREC_FP64], lwc, rtol=1e-12, atol=1e-9)
    # mixed precision against FP64 (erfc form) in log space: the log of the
    # ratio of the per-shift estimates, and the per-sample log-weights.  At
    # these bounds log p is about -14000 and the FP32 steps' errors (chiefly
    # the FP32 inverse normal, relative error up to 4e-7, entering every later
    # conditioning sum) add up over the 1000 variables: measured per-shift
    # |log P_mixed - log P_FP64| up to 0.19 (split BF16, FP32 SIMT) and 0.35
    # (TF32) on 256..4096 points; the bounds below are about twice that.
    lme64 = D.log_mean_exp(lw[L.PREC_FP64])
    bound = {L.PREC_FP32_SPLIT_BF16: 0.4, L.PREC_FP32_SIMT: 0.4, L.PREC_FP32_TF32: 0.8}
    for pr in MIXED:
        assert np.all(np.isfinite(lw[pr])), pr
        dl = np.abs(D.log_mean_exp(lw[pr]) - lme64)
        assert np.all(dl < bound[pr]), (pr, dl)
        assert np.max(np.abs(lw[pr] - lw[L.PREC_FP64])) < 2 * bound[pr] + 0.2, pr


def test_d500_sobol_vs_checker(D, oracle):
    m, R = 1024, 2
    w = W.c2(d=500, m=m, n_reps=R)
    Q = D.QMCData(w.Sigma, w.a, w.b, _opts(D, m, R), qmc_type="Sobol", ushifts=w.ushifts)
    try:
        out = {pr: D.qmc_pnorm(Q, precision=pr, return_reps=True) for pr in [L.PREC_FP64] + MIXED}
        F = Q.C
        Pc, ec, nc, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=m, n_reps=R, max_pts=m, max_abs_err=0.0,
                                          qmc_type=oracle.SOBOL, V=D.sobol_dirnums(499), ushifts=w.ushifts,
                                          sobol_first=Q.sobol_first)
    finally:
        Q.close()
    assert Q.sobol_first == D.sobol_first_index(m)
    np.testing.assert_allclose(out[L.PREC_FP64][3], rc, rtol=1e-12, atol=0)
    assert 0 < Pc < 1e-20  # P of this configuration is tiny but representable
    for pr in MIXED:
        rt = 2e-3 if pr == L.PREC_FP32_TF32 else 2e-4
        np.testing.assert_allclose(out[pr][3], rc, rtol=rt, atol=0, err_msg=f"precision {pr}")

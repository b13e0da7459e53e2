"""Many problems in one call (dbgz_pnorm_batch) against the one-problem path
and the oracle (needs a B200)."""
import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _problems(dims, seed):
    rng = np.random.default_rng(seed)
    out = []
    for d in dims:
        A = rng.standard_normal((d, d + 8))
        S = A @ A.T
        if d % 3 == 0:
            S = W.correlation(S)  # both covariances and correlations
        a = rng.uniform(-2.5, 0.0, d) * np.sqrt(np.diag(S))
        b = rng.uniform(0.0, 2.5, d) * np.sqrt(np.diag(S))
        if d % 4 == 1:
            a[:] = -np.inf
        out.append((S, a, b))
    return out


DIMS = [2, 3, 16, 17, 64, 65, 100, 129, 256, 300, 5, 33]


@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol"])
@pytest.mark.parametrize("prec,rtol", [(L.PREC_FP64, 1e-13), (L.PREC_FP32_SIMT, 1e-6)])
def test_batch_matches_one_problem_path(dbgz, qmc, prec, rtol):
    D = dbgz
    probs = _problems(DIMS, 11)
    opts = D.QMC_opts(m=1000, n_reps=6, max_pts=1000, max_abs_err=0.0)
    rng = np.random.default_rng(5)
    if qmc == "Richtmyer":
        sh = [rng.random((d - 1, 6)) for d in DIMS]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, shifts=sh, precision=prec)
    else:
        ush = [rng.integers(0, 2**63, size=(d - 1, 6), dtype=np.uint64) for d in DIMS]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, ushifts=ush, precision=prec)
    for k, (S, a, b) in enumerate(probs):
        if qmc == "Richtmyer":
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, shifts=sh[k])
        else:
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, ushifts=ush[k])
        P1, e1, _ = D.qmc_pnorm(Q, precision=prec)
        Q.close()
        assert abs(P[k] - P1) <= rtol * abs(P1) + 1e-300, (k, DIMS[k], P[k], P1)
        assert abs(err[k] - e1) <= 1e-6 * abs(e1) + 1e-15


def test_batch_fp64_matches_oracle(dbgz, oracle):
    D = dbgz
    dims = [7, 20, 41]
    probs = _problems(dims, 12)
    rng = np.random.default_rng(6)
    sh = [rng.random((d - 1, 4)) for d in dims]
    opts = D.QMC_opts(m=777, n_reps=4, max_pts=777, max_abs_err=0.0)
    P, _ = D.qmc_pnorm_batch(probs, opts, shifts=sh, precision=L.PREC_FP64)
    for k, (S, a, b) in enumerate(probs):
        F = oracle.cholesky_genz(S, a, b)
        U = oracle.truncate_U(F["U"])
        Po = oracle.qmc_pnorm(U, F["a"], F["b"], m=777, n_reps=4, shifts=sh[k], max_pts=777, max_abs_err=0.0)[0]
        assert abs(P[k] - Po) <= 1e-12 * abs(Po), (k, P[k], Po)


def test_batch_rank_deficient_and_limits(dbgz):
    D = dbgz
    probs = _problems([10, 12, 9], 13)
    v = np.ones(12)
    probs[1] = (np.outer(v, v), -np.ones(12), np.ones(12))  # rank 1
    opts = D.QMC_opts(m=500, n_reps=4, max_pts=500)
    P, err, ranks = D.qmc_pnorm_batch(probs, opts, return_ranks=True, precision=L.PREC_FP64)
    assert ranks[0] == 10 and ranks[2] == 9 and ranks[1] < 12
    assert np.isnan(P[1]) and np.isfinite(P[0]) and np.isfinite(P[2])
    with pytest.raises(L.DbgzError):
        D.qmc_pnorm_batch(probs, opts, precision=L.PREC_FP64)
    big = _problems([513], 14)
    with pytest.raises(L.DbgzError):
        D.qmc_pnorm_batch(big, opts)


def test_batch_fp32_accuracy_many_uneven(dbgz):
    # a C4-shaped batch at reduced size: d ~ U{16..256}, Sobol, FP32 vs FP64
    D = dbgz
    rng = np.random.default_rng(40)
    dims = list(rng.integers(16, 257, size=48))
    probs = _problems(dims, 41)
    opts = D.QMC_opts(m=4096, n_reps=8, max_pts=4096, max_abs_err=0.0)
    ush = [rng.integers(0, 2**63, size=(d - 1, 8), dtype=np.uint64) for d in dims]
    P64, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP64)
    P32, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP32_SIMT)
    assert np.all(np.abs(P32 - P64) <= 2e-6 + 1e-5 * np.abs(P64))


@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol"])
@pytest.mark.parametrize("prec", [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
def test_batch_tensor_core_matches_one_problem_path(dbgz, qmc, prec):
    # problems with d - 1 <= 256 run in the batched tensor-core loop, the rest
    # (d = 300 here) in the SIMT batch loop; each against qmc_pnorm of the same
    # precision (the first dimension's CDF is computed on the device in the
    # batch and on the host in the one-problem path, hence not bit for bit)
    D = dbgz
    dims = DIMS + [257, 250, 130]
    probs = _problems(dims, 17)
    opts = D.QMC_opts(m=1000, n_reps=6, max_pts=1000, max_abs_err=0.0)
    rng = np.random.default_rng(9)
    if qmc == "Richtmyer":
        sh = [rng.random((d - 1, 6)) for d in dims]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, shifts=sh, precision=prec)
    else:
        ush = [rng.integers(0, 2**63, size=(d - 1, 6), dtype=np.uint64) for d in dims]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, ushifts=ush, precision=prec)
    for k, (S, a, b) in enumerate(probs):
        if qmc == "Richtmyer":
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, shifts=sh[k])
        else:
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, ushifts=ush[k])
        P1, e1, _ = D.qmc_pnorm(Q, precision=prec)
        P64, _, _ = D.qmc_pnorm(Q, precision=L.PREC_FP64)
        Q.close()
        assert abs(P[k] - P1) <= 1e-6 * abs(P1) + 1e-12, (k, dims[k], P[k], P1)
        assert abs(P[k] - P64) <= 2e-6 + 1e-5 * abs(P64), (k, dims[k], P[k], P64)


def test_batch_tensor_core_many_problems(dbgz):
    # more problems than CTAs, all single-phase: the item list spans problems
    D = dbgz
    rng = np.random.default_rng(44)
    dims = list(rng.integers(2, 258, size=400))
    probs = _problems(dims, 45)
    opts = D.QMC_opts(m=512, n_reps=4, max_pts=512, max_abs_err=0.0)
    ush = [rng.integers(0, 2**63, size=(d - 1, 4), dtype=np.uint64) for d in dims]
    P64, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP64)
    Pt, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP32_SPLIT_BF16)
    Ps, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP32_SIMT)
    assert np.all(np.abs(Pt - P64) <= 2e-6 + 1e-5 * np.abs(P64))
    assert np.all(np.abs(Pt - Ps) <= 2e-6 + 1e-5 * np.abs(Ps))

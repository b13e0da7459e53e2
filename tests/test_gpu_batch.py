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


# "Sobol2048": Sobol from index 2048, a multiple of 128 (the loops' staged
# integers) with a partial last tile (m = 1000); "Sobol": from 2m = 2000
@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol", "Sobol2048"])
@pytest.mark.parametrize("prec,rtol", [(L.PREC_FP64, 1e-13), (L.PREC_FP32_SIMT, 1e-6)])
def test_batch_matches_one_problem_path(dbgz, qmc, prec, rtol):
    D = dbgz
    probs = _problems(DIMS, 11)
    opts = D.QMC_opts(m=1000, n_reps=6, max_pts=1000, max_abs_err=0.0)
    rng = np.random.default_rng(5)
    first = 2048 if qmc == "Sobol2048" else None
    qmc = qmc[:5] if first else qmc
    if qmc == "Richtmyer":
        sh = [rng.random((d - 1, 6)) for d in DIMS]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, shifts=sh, precision=prec)
    else:
        ush = [rng.integers(0, 2**63, size=(d - 1, 6), dtype=np.uint64) for d in DIMS]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, ushifts=ush, precision=prec, sobol_first=first)
    for k, (S, a, b) in enumerate(probs):
        if qmc == "Richtmyer":
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, shifts=sh[k])
        else:
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, ushifts=ush[k], sobol_first=first)
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


@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol", "Sobol2048"])
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
    first = 2048 if qmc == "Sobol2048" else None
    qmc = qmc[:5] if first else qmc
    if qmc == "Richtmyer":
        sh = [rng.random((d - 1, 6)) for d in dims]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, shifts=sh, precision=prec)
    else:
        ush = [rng.integers(0, 2**63, size=(d - 1, 6), dtype=np.uint64) for d in dims]
        P, err = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, ushifts=ush, precision=prec, sobol_first=first)
    for k, (S, a, b) in enumerate(probs):
        if qmc == "Richtmyer":
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, shifts=sh[k])
        else:
            Q = D.QMCData(S, a, b, opts, qmc_type=qmc, ushifts=ush[k], sobol_first=first)
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


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32_SIMT, L.PREC_FP32_SPLIT_BF16])
@pytest.mark.parametrize("qmc", ["Richtmyer", "Sobol"])
def test_batch_plan_graph_matches_one_shot(dbgz, prec, qmc):
    # the graph of a plan runs the same kernels on the same inputs: the same
    # bits as the one-shot call, run after run, with new inputs each run
    D = dbgz
    dims = [40, 7, 200, 33, 300, 16]
    opts = D.QMC_opts(m=700, n_reps=5, max_pts=700, max_abs_err=0.0)
    plan = D.BatchPlan(dims, opts, qmc_type=qmc, precision=prec)
    try:
        info = plan.info()
        assert info["tensor_problems"] + info["simt_items"] > 0 and info["kernels_per_run"] >= 3
        for seed in (21, 22):
            probs = _problems(dims, seed)
            rng = np.random.default_rng(seed)
            if qmc == "Richtmyer":
                sh = [rng.random((d - 1, 5)) for d in dims]
                P1, e1 = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, shifts=sh, precision=prec)
            else:
                sh = [rng.integers(0, 2**63, size=(d - 1, 5), dtype=np.uint64) for d in dims]
                P1, e1 = D.qmc_pnorm_batch(probs, opts, qmc_type=qmc, ushifts=sh, precision=prec)
            plan.fill(probs, sh)
            P, err = plan.run()
            assert np.array_equal(P, P1) and np.array_equal(err, e1), (P - P1, err - e1)
    finally:
        plan.close()


def test_batch_input_checks_on_device(dbgz):
    D = dbgz
    dims = [12, 30, 9]
    opts = D.QMC_opts(m=256, n_reps=4, max_pts=256)
    probs = _problems(dims, 31)
    rng = np.random.default_rng(3)
    sh = [rng.random((d - 1, 4)) for d in dims]
    bad_S = [(S.copy(), a, b) for S, a, b in probs]
    bad_S[1][0][3, 4] = np.nan
    bad_ab = [(S, a.copy(), b.copy()) for S, a, b in probs]
    bad_ab[2][1][0] = bad_ab[2][2][0] + 1.0  # a > b
    bad_sh = [x.copy() for x in sh]
    bad_sh[0][2, 1] = 1.5
    for pr, shx, code in ((bad_S, sh, L.ERR_NONFINITE_INPUT), (bad_ab, sh, L.ERR_NONFINITE_INPUT),
                          (probs, bad_sh, L.ERR_INVALID_ARGUMENT)):
        with pytest.raises(L.DbgzError) as ei:
            D.qmc_pnorm_batch(pr, opts, shifts=shx, precision=L.PREC_FP32_SIMT)
        assert ei.value.status == code
    plan = D.BatchPlan(dims, opts, precision=L.PREC_FP32_SPLIT_BF16)
    try:
        plan.fill(bad_S, sh)
        with pytest.raises(L.DbgzError) as ei:
            plan.run()
        assert ei.value.status == L.ERR_NONFINITE_INPUT
        plan.fill(probs, sh)  # the plan stays usable
        P, _ = plan.run()
        P1, _ = D.qmc_pnorm_batch(probs, opts, shifts=sh, precision=L.PREC_FP32_SPLIT_BF16)
        assert np.array_equal(P, P1)
    finally:
        plan.close()


def test_batch_autotune_table_and_results(dbgz):
    # own context: the table is per context
    D = dbgz
    ctx = D.Context(0)
    try:
        opts = D.QMC_opts(m=1024, n_reps=4, max_pts=1024, max_abs_err=0.0)
        eng0, it0, tuned0 = D.batch_tuning(L.PREC_FP32_SPLIT_BF16, "Sobol", context=ctx)
        assert not tuned0 and eng0[24] == 0 and eng0[25] == 1 and eng0[258] == 0 and it0[100] == 1024
        eng, items = D.batch_autotune(opts, L.PREC_FP32_SPLIT_BF16, "Sobol", context=ctx)
        assert set(np.unique(eng[2:])) <= {0, 1} and np.all(eng[258:] == 0)
        assert set(np.unique(items[2:])) <= {256, 1024, 4096}
        eng2, items2, tuned = D.batch_tuning(L.PREC_FP32_SPLIT_BF16, "Sobol", context=ctx)
        assert tuned and np.array_equal(eng2[2:], eng[2:]) and np.array_equal(items2[2:], items[2:])
        dims = [10, 20, 60, 130, 250, 400]
        probs = _problems(dims, 51)
        rng = np.random.default_rng(52)
        ush = [rng.integers(0, 2**63, size=(d - 1, 4), dtype=np.uint64) for d in dims]
        Pt, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP32_SPLIT_BF16,
                                  context=ctx)
        P64, _ = D.qmc_pnorm_batch(probs, opts, qmc_type="Sobol", ushifts=ush, precision=L.PREC_FP64, context=ctx)
        assert np.all(np.abs(Pt - P64) <= 2e-6 + 1e-5 * np.abs(P64))
    finally:
        ctx.close()

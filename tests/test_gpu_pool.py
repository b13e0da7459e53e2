"""The context's stream-ordered buffer cache (needs a B200).

A problem built on recycled buffers must give bit-identical results to one
built on fresh buffers; freed problems' buffers stay cached until
dbgz_release_cached; a context with live problems refuses to be destroyed."""
import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _case(D, ctx, n, seed, prec):
    rng = np.random.default_rng(seed)
    S = W.rand_spd(n, 1.0, rng)
    lo, up = W.bounds_quarter(S)
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=3000, n_reps=6, max_pts=3000, max_abs_err=0.0),
                  shifts=rng.random((n - 1, 6)), context=ctx)
    r = D.qmc_pnorm(Q, precision=prec, return_reps=True)
    g = D.qmc_pnorm_grad(Q, precision=prec) if prec != L.PREC_FP64 or n < 200 else None
    U = Q.C.U.copy()
    Q.close()
    return r, g, U


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32_SPLIT_BF16])
def test_recycled_buffers_give_identical_results(dbgz, prec):
    D = dbgz
    ctx = D.Context(0)
    try:
        assert ctx.release_cached() == 0
        r1, g1, U1 = _case(D, ctx, 150, 7, prec)
        # a different problem in between dirties the recycled blocks
        _case(D, ctx, 90, 8, prec)
        r2, g2, U2 = _case(D, ctx, 150, 7, prec)
        assert np.array_equal(U1, U2)
        assert r1[0] == r2[0] and np.array_equal(r1[3], r2[3])
        if g1 is not None:
            for x, y in zip(g1[3:], g2[3:]):
                assert np.array_equal(x, y)
        assert ctx.release_cached() > 0
        assert ctx.release_cached() == 0
    finally:
        ctx.close()


def test_destroy_refuses_live_problems(dbgz):
    D = dbgz
    ctx = D.Context(0)
    S = W.rand_spd(20, 1.0, np.random.default_rng(1))
    Q = D.QMCData(S, -np.ones(20), np.ones(20), D.QMC_opts(m=256, n_reps=2, max_pts=256), context=ctx)
    assert L.lib().dbgz_destroy(ctx.handle) == L.ERR_INVALID_ARGUMENT
    Q.close()
    ctx.close()
    assert ctx.handle is None

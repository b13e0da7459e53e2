"""Adjoint of the estimator (dbgz_pnorm_grad) against central finite
differences on common QMC points (needs a B200).

Finite differences perturb the factor U and the permuted, scaled bounds
directly, through the allocation-free FP64 pass, so the pivot order stays
frozen and every evaluation uses the same points and shifts; the gradient is
then an exact derivative of the same estimate."""
import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L

pytestmark = pytest.mark.gpu


class FdPass:
    """P(U, a, b) on the first pass's points, through dbgz_pnorm_pass_noalloc."""

    def __init__(self, Q):
        import torch
        self.torch = torch
        self.Q = Q
        self.n = Q.n
        self.m = Q.opts.m
        self.n_reps = Q.opts.n_reps
        dev = torch.device("cuda", 0)
        self.dev = dev
        f = lambda x: torch.from_numpy(np.ascontiguousarray(np.ravel(x, order="F"), dtype=np.float64)).to(dev)
        import dbgenzpaper_b200 as D
        self.q = f(D.get_sqrt_primes(self.n - 1))
        self.sh = f(Q.shifts)
        self.out = torch.zeros(self.n_reps, dtype=torch.float64, device=dev)
        self.f = f

    def __call__(self, U, a, b):
        Ud, ad, bd = self.f(U), self.f(a), self.f(b)
        st = L.lib().dbgz_pnorm_pass_noalloc(self.n, Ud.data_ptr(), ad.data_ptr(), bd.data_ptr(), self.q.data_ptr(),
                                             self.sh.data_ptr(), self.m, self.n_reps, 0, self.out.data_ptr(),
                                             self.torch.cuda.current_stream(self.dev).cuda_stream)
        assert st == 0
        self.torch.cuda.synchronize(self.dev)
        return float(self.out.mean().item())


def _problem(D, n, seed, a_inf=False):
    rng = np.random.default_rng(seed)
    S = W.rand_spd(n, 1.0, rng)
    lo, up = W.bounds_quarter(S)
    if a_inf:
        lo = np.full(n, -np.inf)
        up = rng.uniform(0.0, 2.0, n) * np.sqrt(np.diag(S))
    sh = rng.random((n - 1, 4))
    return D.QMCData(S, lo, up, D.QMC_opts(m=384, n_reps=4, max_pts=384, max_abs_err=0.0), shifts=sh)


@pytest.mark.parametrize("n,a_inf", [(10, False), (70, False), (40, True)])
def test_fp64_gradient_matches_finite_differences(dbgz, n, a_inf):
    D = dbgz
    Q = _problem(D, n, 1000 + n, a_inf)
    P, err, npts, da, db, dU = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
    P1 = D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]
    assert abs(P - P1) <= 1e-14 * abs(P1) + 1e-300 and npts == 384
    F = Q.C
    U, a, b, perm, sv = F.U.copy(), F.a.copy(), F.b.copy(), F.perm, F.scale_vec
    fd = FdPass(Q)
    P0 = fd(U, a, b)
    assert abs(P0 - P) <= 1e-12 * abs(P)
    rng = np.random.default_rng(n)
    h = 1e-6
    # bounds: dP/db_perm[t] = dP/db_orig[perm[t]] * scale[perm[t]]
    for t in rng.choice(n, size=min(n, 6), replace=False):
        for which, g in (("b", db), ("a", da)):
            if which == "a" and a_inf:
                continue
            vp, vm = (a.copy(), a.copy()) if which == "a" else (b.copy(), b.copy())
            vp[t] += h
            vm[t] -= h
            if which == "a":
                fdv = (fd(U, vp, b) - fd(U, vm, b)) / (2 * h)
            else:
                fdv = (fd(U, a, vp) - fd(U, a, vm)) / (2 * h)
            an = g[perm[t]] * sv[perm[t]]
            assert abs(an - fdv) <= 2e-6 * max(abs(fdv), abs(P)) + 1e-12, (which, t, an, fdv)
    # factor entries, off-diagonal and diagonal
    pairs = [(l, t) for t in range(1, n) for l in range(t)]
    idx = rng.choice(len(pairs), size=min(8, len(pairs)), replace=False)
    for (l, t) in [pairs[i] for i in idx] + [(0, 0), (n - 1, n - 1), (n // 2, n // 2)]:
        Up, Um = U.copy(), U.copy()
        Up[l, t] += h
        Um[l, t] -= h
        fdv = (fd(Up, a, b) - fd(Um, a, b)) / (2 * h)
        assert abs(dU[l, t] - fdv) <= 2e-6 * max(abs(fdv), abs(P)) + 1e-12, (l, t, dU[l, t], fdv)
    assert np.all(np.tril(dU, -1) == 0)


@pytest.mark.parametrize("prec,tol", [(L.PREC_FP32_SIMT, 2e-3), (L.PREC_FP32_SPLIT_BF16, 2e-3),
                                      (L.PREC_FP32_TF32, 2e-2)])
@pytest.mark.parametrize("n", [50, 300, 700])
def test_fp32_gradients_close_to_fp64(dbgz, prec, tol, n):
    # n = 300 crosses the tensor loop's 256-wide phases in both directions;
    # n = 700 gives the factor-gradient GEMM a 6 x 3 grid of 128 x 256 tiles
    # with partial tiles at both edges
    D = dbgz
    Q = _problem(D, n, 2000 + n)
    P64, _, _, da64, db64, dU64 = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
    P, _, _, da, db, dU = D.qmc_pnorm_grad(Q, precision=prec)
    assert abs(P - P64) <= 1e-4 * abs(P64) + 1e-6
    for g, g64 in ((da, da64), (db, db64), (dU, dU64)):
        assert np.linalg.norm(g - g64) <= tol * np.linalg.norm(g64), (np.linalg.norm(g - g64) / np.linalg.norm(g64))


def _sigma_problem(n, seed, finite_a=True):
    rng = np.random.default_rng(seed)
    R = W.correlation(W.rand_spd(n, 1.0, rng))
    s = rng.uniform(0.5, 2.0, n)
    S = R * np.outer(s, s)  # a covariance, not a correlation: exercises the scaling
    # bounds without ties in the first pivot scores (a symmetric design such
    # as +-k sqrt(S_ii) makes every first score equal, and a perturbation of
    # Sigma_ii then moves the pivot order)
    lo, up = -rng.uniform(0.3, 2.0, n) * s, rng.uniform(0.3, 2.0, n) * s
    if not finite_a:
        lo = np.full(n, -np.inf)
    return S, lo, up, rng.random((n - 1, 4))


def _P(D, S, lo, up, sh):
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=384, n_reps=4, max_pts=384, max_abs_err=0.0), shifts=sh)
    P = D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]
    perm = Q.C.perm.copy()
    Q.close()
    return P, perm


@pytest.mark.parametrize("n,finite_a", [(12, True), (48, False)])
def test_sigma_gradient_matches_finite_differences(dbgz, n, finite_a):
    D = dbgz
    S, lo, up, sh = _sigma_problem(n, 3000 + n, finite_a)
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=384, n_reps=4, max_pts=384, max_abs_err=0.0), shifts=sh)
    P, _, _, da, db, G = D.qmc_pnorm_grad_sigma(Q, precision=L.PREC_FP64)
    perm0 = Q.C.perm.copy()
    Q.close()
    assert np.allclose(G, G.T, rtol=1e-12, atol=1e-14 * np.abs(G).max())
    rng = np.random.default_rng(n)
    h = 1e-6
    pairs = [(i, i) for i in rng.choice(n, 3, replace=False)]
    pairs += [tuple(sorted(rng.choice(n, 2, replace=False))) for _ in range(6)]
    checked = 0
    for i, j in pairs:
        E = np.zeros((n, n))
        E[i, j] = E[j, i] = h
        Pp, pp = _P(D, S + E, lo, up, sh)
        Pm, pm = _P(D, S - E, lo, up, sh)
        if not (np.array_equal(pp, perm0) and np.array_equal(pm, perm0)):
            continue  # the pivot order moved: not a derivative of the same estimate
        fd = (Pp - Pm) / (2 * h)
        an = G[i, i] if i == j else 2 * G[i, j]
        assert abs(an - fd) <= 2e-6 * max(abs(fd), abs(P)) + 1e-11, (i, j, an, fd)
        checked += 1
    assert checked >= len(pairs) - 1
    # bounds at fixed Sigma through the public gradient
    for i in rng.choice(n, 3, replace=False):
        e = np.zeros(n)
        e[i] = h
        fd = (_P(D, S, lo, up + e, sh)[0] - _P(D, S, lo, up - e, sh)[0]) / (2 * h)
        assert abs(db[i] - fd) <= 2e-6 * max(abs(fd), abs(P)) + 1e-11


def test_factor_model_dB(dbgz):
    # Sigma = B B' + diag(psi): dP/dB = 2 G B, checked by central differences on B
    D = dbgz
    rng = np.random.default_rng(77)
    n, k = 40, 3
    B = rng.normal(0, 0.5, (n, k))
    psi = rng.uniform(0.2, 1.0, n)
    S = B @ B.T + np.diag(psi)
    lo = np.full(n, -np.inf)
    up = rng.uniform(0.0, 2.0, n) * np.sqrt(np.diag(S))
    sh = rng.random((n - 1, 4))
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=384, n_reps=4, max_pts=384, max_abs_err=0.0), shifts=sh)
    P, _, _, _, _, G = D.qmc_pnorm_grad_sigma(Q, precision=L.PREC_FP64)
    # the host-side entry point on the outputs of qmc_pnorm_grad gives the same matrix
    _, _, _, da, db, dU = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
    assert np.array_equal(D.sigma_adjoint(Q, dU, da, db), G)
    perm0 = Q.C.perm.copy()
    Q.close()
    dB = 2 * G @ B
    h = 1e-6
    for i, j in [(0, 0), (5, 1), (n - 1, 2), (17, 0)]:
        Bp, Bm = B.copy(), B.copy()
        Bp[i, j] += h
        Bm[i, j] -= h
        Pp, pp = _P(D, Bp @ Bp.T + np.diag(psi), lo, up, sh)
        Pm, pm = _P(D, Bm @ Bm.T + np.diag(psi), lo, up, sh)
        assert np.array_equal(pp, perm0) and np.array_equal(pm, perm0)
        fd = (Pp - Pm) / (2 * h)
        assert abs(dB[i, j] - fd) <= 2e-6 * max(abs(fd), abs(P)) + 1e-11, (i, j, dB[i, j], fd)


def test_fp32_sigma_gradient_close_to_fp64(dbgz):
    D = dbgz
    S, lo, up, sh = _sigma_problem(200, 4200)
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=2048, n_reps=4, max_pts=2048, max_abs_err=0.0), shifts=sh)
    G64 = D.qmc_pnorm_grad_sigma(Q, precision=L.PREC_FP64)[5]
    G = D.qmc_pnorm_grad_sigma(Q, precision=L.PREC_FP32_SPLIT_BF16)[5]
    assert np.linalg.norm(G - G64) <= 3e-3 * np.linalg.norm(G64)


@pytest.mark.parametrize("prec,rtol", [(L.PREC_FP64, 1e-11), (L.PREC_FP32_SPLIT_BF16, 1e-4)])
def test_chunked_gradient_matches_one_chunk(dbgz, prec, rtol):
    # a small state budget splits the samples into chunks of tiles: the same
    # estimate, and the same gradient up to the summation grouping
    D = dbgz
    ctx = D.Context(0)
    try:
        rng = np.random.default_rng(90)
        n = 120
        S = W.rand_spd(n, 1.0, rng)
        lo, up = W.bounds_quarter(S)
        opts = D.QMC_opts(m=3000, n_reps=5, max_pts=3000, max_abs_err=0.0)
        Q = D.QMCData(S, lo, up, opts, shifts=rng.random((n - 1, 5)), context=ctx)
        r1 = D.qmc_pnorm_grad(Q, precision=prec)
        ctx.set_state_budget(3 << 20)  # a few tiles per chunk
        r2 = D.qmc_pnorm_grad(Q, precision=prec)
        P1 = D.qmc_pnorm(Q, precision=prec)[0]
        Q.close()
        assert r1[0] == r2[0] and r1[1] == r2[1] and abs(r1[0] - P1) <= 1e-12 * P1
        for x, y in zip(r1[3:], r2[3:]):
            assert np.linalg.norm(y) > 0
            assert np.linalg.norm(x - y) <= rtol * np.linalg.norm(y)
    finally:
        ctx.close()


def _banded(n, seed):
    rng = np.random.default_rng(seed)
    idx = np.arange(n)
    dist = np.abs(idx[:, None] - idx[None, :])
    S = 0.8 ** dist + 0.3 * (dist == 1) + 0.5 * np.eye(n)
    up = rng.uniform(-0.5, 2.5, n)
    lo = np.minimum(-rng.uniform(0.5, 2.5, n), up - 0.3)
    return S, lo, up, rng.random((n - 1, 4))


def _banded_problem(D, S, lo, up, sh, band, m=512, context=None, sobol=False):
    # sobol: Sobol points from index 2048 (a multiple of 128: the loops'
    # staged integers), random shifts drawn from sh's values
    kw = dict(qmc_type="Richtmyer", shifts=sh)
    if sobol:
        kw = dict(qmc_type="Sobol", ushifts=(sh * 2.0**63).astype(np.uint64), sobol_first=2048)
    Q = D.QMCDataSparse(S, lo, up, D.QMC_opts(m=m, n_reps=4, max_pts=m, max_abs_err=0.0),
                        context=context, **kw)
    Q.truncate_band(band)
    return Q


def _Pband(D, S, lo, up, sh, band, m=512, sobol=False):
    Q = _banded_problem(D, S, lo, up, sh, band, m=m, sobol=sobol)
    P = D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]
    Q.close()
    return P


@pytest.mark.parametrize("qmc,m", [("Richtmyer", 512), ("Sobol", 500)])
def test_banded_gradient_matches_finite_differences(dbgz, qmc, m):
    # the banded path (classic factor, no pivoting) against central
    # differences of the banded estimate in the original bounds; Sobol: the
    # adjoint takes the staged integers (partial last tile)
    D = dbgz
    n, band = 90, 6
    sob = qmc == "Sobol"
    S, lo, up, sh = _banded(n, 91)
    Q = _banded_problem(D, S, lo, up, sh, band, m=m, sobol=sob)
    P, _, _, da, db, dU = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
    assert dU is None
    assert abs(P - D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]) <= 1e-14 * P
    Q.close()
    h = 1e-6
    rng = np.random.default_rng(3)
    for i in rng.choice(n, 6, replace=False):
        e = np.zeros(n)
        e[i] = h
        fdb = (_Pband(D, S, lo, up + e, sh, band, m, sob) - _Pband(D, S, lo, up - e, sh, band, m, sob)) / (2 * h)
        fda = (_Pband(D, S, lo + e, up, sh, band, m, sob) - _Pband(D, S, lo - e, up, sh, band, m, sob)) / (2 * h)
        assert abs(db[i] - fdb) <= 2e-6 * max(abs(fdb), abs(P)) + 1e-12, (i, db[i], fdb)
        assert abs(da[i] - fda) <= 2e-6 * max(abs(fda), abs(P)) + 1e-12, (i, da[i], fda)


def test_banded_gradient_chunked_and_fp32(dbgz):
    D = dbgz
    ctx = D.Context(0)
    try:
        n, band = 700, 40  # the anti-transposed CSC in a 64-slot shared-memory ring
        S, lo, up, sh = _banded(n, 92)
        Q = _banded_problem(D, S, lo, up, sh, band, m=1024, context=ctx)
        r64 = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
        r32 = D.qmc_pnorm_grad(Q, precision=L.PREC_FP32_SIMT)
        ctx.set_state_budget(8 << 20)
        r64c = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
        P64 = D.qmc_pnorm(Q, precision=L.PREC_FP64)[0]
        Q.close()
        assert r64[0] == r64c[0] and abs(r64[0] - P64) <= 1e-14 * P64
        for x, y in zip(r64c[3:5], r64[3:5]):
            assert np.linalg.norm(x - y) <= 1e-11 * np.linalg.norm(y)
        assert abs(r32[0] - r64[0]) <= 1e-5 * r64[0] + 1e-7
        for x, y in zip(r32[3:5], r64[3:5]):
            assert np.linalg.norm(x - y) <= 2e-3 * np.linalg.norm(y)
    finally:
        ctx.close()


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32_SIMT])
@pytest.mark.parametrize("qmc,seg,n,band", [("Richtmyer", 32, 150, 6), ("Sobol", 64, 300, 40), ("Sobol", 256, 700, 40),
                                            ("Richtmyer", 5, 40, 3), ("Richtmyer", 100, 90, 6)])
def test_banded_gradient_checkpoints_same_bits(dbgz, prec, qmc, seg, n, band):
    # dimension checkpoints (a checkpoint every `seg` dimensions, each segment
    # recomputed before the adjoint sweeps it) against storing the whole
    # forward state: the same kernels on the same values, so P and the
    # gradients are the same bits; also with the samples split in chunks
    D = dbgz
    ctx = D.Context(0)
    try:
        S, lo, up, sh = _banded(n, 93 + n)
        Q = _banded_problem(D, S, lo, up, sh, band, m=600, sobol=qmc == "Sobol", context=ctx)
        ctx.set_grad_checkpoints(0)
        full = D.qmc_pnorm_grad(Q, precision=prec)
        ctx.set_grad_checkpoints(seg)
        ck = D.qmc_pnorm_grad(Q, precision=prec)
        ctx.set_state_budget(2 << 20)  # several chunks of tiles
        ckc = D.qmc_pnorm_grad(Q, precision=prec)
        Q.close()
        assert ck[0] == full[0] and ck[1] == full[1]
        assert np.array_equal(ck[3], full[3]) and np.array_equal(ck[4], full[4])
        assert ckc[0] == full[0]
        for x, y in zip(ckc[3:5], full[3:5]):
            assert np.linalg.norm(x - y) <= 1e-11 * np.linalg.norm(y)
    finally:
        ctx.close()

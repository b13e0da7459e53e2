"""CUDA path against the CPU checker and the golden fixtures (needs a B200).

Bars: bit-exact for the factorisation (U, pivot permutation, permuted
bounds) and the point sets; FP64 probabilities within 1e-12 relative of the
checker (the two use different erf/erfinv implementations and summation
orders); FP32 modes within the tolerances written in each test."""
import ctypes as C
import os

import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L
from oracle import kat

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def D(dbgz):
    dbgz.get_context(0)
    return dbgz


def _spd(n, seed, jitter=1.0):
    return W.rand_spd(n, jitter, np.random.default_rng(seed))


# ---------------------------------------------------------------- factor ---
@pytest.mark.parametrize("n,bs1,bs2,seed", [(7, 64, 512, 1), (64, 64, 512, 2), (130, 16, 64, 3),
                                            (600, 64, 512, 4), (300, 8, 32, 5)])
def test_cholesky_genz_bitexact(D, oracle, n, bs1, bs2, seed):
    S = _spd(n, seed)
    rng = np.random.default_rng(seed)
    a = rng.uniform(-3, 0, n)
    b = rng.uniform(0, 3, n)
    a[::5] = -np.inf
    G = D.cholesky_genz(S, a, b, bs1, bs2)
    F = oracle.cholesky_genz(S, a, b, bs1, bs2)
    assert G.rank == F["rank"] == n
    assert np.array_equal(G.perm, F["perm"])
    assert np.array_equal(G.U, F["U"])  # whole matrix, lower-triangle scratch included
    assert np.array_equal(G.a, F["a"]) and np.array_equal(G.b, F["b"])
    assert np.array_equal(G.scale_vec, F["scale_vec"])


def test_cholesky_genz_reference_case(D, oracle):
    # test/runtests.jl:15-36 at n = 1024 (three bs2 panels with bs2 = 512? no: 2)
    rng = np.random.default_rng(101)
    n = 1024
    A = rng.random((n, n))
    Cm = A @ A.T + 100.0 * np.eye(n)
    G = D.cholesky_genz(Cm, -np.ones(n), np.ones(n), 64, 512)
    F = oracle.cholesky_genz(Cm, -np.ones(n), np.ones(n), 64, 512)
    assert np.array_equal(G.perm, F["perm"]) and np.array_equal(G.U, F["U"])
    d = np.sqrt(np.diag(Cm))
    Ct = Cm / np.outer(d, d)
    U = np.triu(G.U)
    assert np.max(np.abs(Ct[np.ix_(G.perm, G.perm)] - U.T @ U)) < 1e-10


def test_cholesky_genz_ties_pick_first_index(D, oracle):
    # equicorrelated Sigma with equal bounds: every score ties exactly
    n = 40
    S = W.fixed_dense(n)
    lo, up = W.bounds_quarter(S)
    G = D.cholesky_genz(S, lo, up, 8, 16)
    F = oracle.cholesky_genz(S, lo, up, 8, 16)
    assert np.array_equal(G.perm, F["perm"]) and np.array_equal(G.U, F["U"])


def test_cholesky_genz_near_ties(D, oracle):
    # random covariances with the reference's symmetric bound design: the
    # checker's pivot log shows a step whose two best scores tie exactly (and
    # others within 1e-9), where any other rounding could flip the pivot; the
    # GPU factorisation (the same deterministic FP64 arithmetic) still agrees
    # bit for bit
    near = 0
    for seed in range(4):
        S = _spd(120, 50 + seed)
        lo, up = W.bounds_quarter(S)
        F = oracle.cholesky_genz(S, lo, up, 32, 64, margins=True)
        G = D.cholesky_genz(S, lo, up, 32, 64)
        near += int(np.sum(F["margins"] < 1e-12))
        assert np.array_equal(G.perm, F["perm"]) and np.array_equal(G.U, F["U"])
    assert near > 0  # the case is exercised


def test_cholesky_genz_rank_deficient(D, oracle):
    rng = np.random.default_rng(9)
    B = rng.standard_normal((20, 5))
    S = B @ B.T
    G = D.cholesky_genz(S, -np.ones(20), np.ones(20), 8, 16)
    F = oracle.cholesky_genz(S, -np.ones(20), np.ones(20), 8, 16)
    assert G.rank == F["rank"] < 20
    k = G.rank
    assert np.array_equal(G.perm, F["perm"])
    assert np.array_equal(np.triu(G.U)[:k, :k], np.triu(F["U"])[:k, :k])


@pytest.mark.parametrize("n,bs", [(100, 8), (100, 16), (100, 32), (100, 64), (300, 128)])
def test_cholesky_classic_bitexact(D, oracle, n, bs):
    # test/runtests.jl:38-59
    rng = np.random.default_rng(102)
    A = rng.random((n, n))
    Cm = A @ A.T + 100.0 * np.eye(n)
    G = D.cholesky_classic(Cm, -np.ones(n), np.ones(n), bs, bs, bs, bs)
    F = oracle.cholesky_classic(Cm, -np.ones(n), np.ones(n), bs, bs, bs, bs)
    assert np.array_equal(np.triu(G.U), np.triu(F["U"]))
    d = np.sqrt(np.diag(Cm))
    U = np.triu(G.U)
    assert np.max(np.abs(Cm / np.outer(d, d) - U.T @ U)) < 1e-10


# ---------------------------------------------------------------- points ---
@pytest.mark.parametrize("n0", [0, 10_000, 2**20])
def test_richtmyer_bitexact(D, oracle, n0):
    q = D.get_sqrt_primes(50)
    assert np.array_equal(D.richtmyer_mat(1000, q, n0), oracle.richtmyer_mat(1000, q, n0))


@pytest.mark.parametrize("first", [0, 2048, 12345])
def test_sobol_bitexact(D, oracle, first):
    V = D.sobol_dirnums(20)
    assert np.array_equal(D.sobol_mat(4096, V, first), oracle.sobol_points(V, first, 4096))


# ------------------------------------------------------------- integrate ---
def _case(z, c):
    return {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(c + "/")}


def _from_case(D, g, T=np.float64, precision=None):
    opts = D.QMC_opts(T, m=int(g["m"]), n_reps=int(g["n_reps"]), max_pts=int(g["max_pts"]),
                      max_abs_err=0.0, chol_block_size=int(g["bs1"]), chol_block_size2=int(g["bs2"]))
    kw = dict(precision=precision, cdf_form=int(g["cdf_form"]))
    if int(g["qmc_type"]) == 0:
        kw.update(qmc_type="Richtmyer", shifts=g["shifts"])
    else:
        kw.update(qmc_type="Sobol", ushifts=g["ushifts"], sobol_dirnums=g["V"],
                  sobol_first=int(g["sobol_first"]))
    cls = D.QMCDataSparse if int(g["sparse"]) else D.QMCData
    return cls(g["Sigma"], g["a_in"], g["b_in"], opts, **kw)


DENSE_CASES = ["c1", "spd8", "sobol40", "erfc130"]


@pytest.mark.parametrize("c", DENSE_CASES)
def test_pnorm_fp64_matches_fixture(D, c):
    z = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    g = _case(z, c)
    Q = _from_case(D, g)
    F = Q.C
    assert np.array_equal(F.perm, g["perm"]) and np.array_equal(np.triu(F.U), np.triu(g["U"]))
    P, err, npts, reps = D.qmc_pnorm(Q, return_reps=True)
    assert npts == int(g["n_pts"])
    np.testing.assert_allclose(reps, g["reps"], rtol=1e-12, atol=1e-300)
    assert abs(P - float(g["P"])) <= 1e-12 * abs(float(g["P"]))
    assert abs(err - float(g["err"])) <= 1e-9 * abs(float(g["err"])) + 1e-15


@pytest.mark.parametrize("c", DENSE_CASES)
def test_pnorm_fp32_simt_close_to_fp64(D, c):
    # FP32 numerics (FP64 weight product): |P - P64| <= 2e-6 + 1e-5 |P|
    z = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    g = _case(z, c)
    Q = _from_case(D, g, np.float32, precision=L.PREC_FP32_SIMT)
    P, err, npts, reps = D.qmc_pnorm(Q, return_reps=True)
    P64 = float(g["P"])
    assert abs(P - P64) <= 2e-6 + 1e-5 * abs(P64), (P, P64)
    np.testing.assert_allclose(reps, g["reps"], rtol=1e-4, atol=2e-6)


def test_pnorm_fp64_multi_group_vs_checker(D, oracle):
    # d = 300 crosses several 64-wide groups; m not a multiple of the tile
    n = 300
    S = _spd(n, 300)
    lo, up = W.bounds_quarter(S)
    sh = np.random.default_rng(300).random((n - 1, 4))
    opts = D.QMC_opts(m=700, n_reps=4, max_pts=1400, max_abs_err=0.0)
    Q = D.QMCData(S, lo, up, opts, shifts=sh)
    P, err, npts, reps = D.qmc_pnorm(Q, return_reps=True)
    F = Q.C
    Pc, ec, nc, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=700, n_reps=4, shifts=sh, max_pts=1400,
                                      max_abs_err=0.0)
    assert npts == nc == 1400
    np.testing.assert_allclose(reps, rc, rtol=1e-12)


def test_second_call_continues_sequence(D, oracle):
    # qmc_pnorm! twice on the same QMCData: the generator state persists
    n = 20
    S = _spd(n, 20)
    lo, up = W.bounds_quarter(S)
    sh = np.random.default_rng(20).random((n - 1, 3))
    opts = D.QMC_opts(m=256, n_reps=3, max_pts=512, max_abs_err=0.0)
    Q = D.QMCData(S, lo, up, opts, shifts=sh)
    D.qmc_pnorm(Q)
    P2, _, n2, r2 = D.qmc_pnorm(Q, return_reps=True)
    F = Q.C
    _, _, _, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=256, n_reps=3, shifts=sh, max_pts=512,
                                   max_abs_err=0.0, gen_base0=256)
    assert n2 == 512
    np.testing.assert_allclose(r2, rc, rtol=1e-12)


def test_distributions_variant_gpu(D, oracle):
    S = _spd(30, 31)
    lo, up = W.bounds_quarter(S)
    sh = np.random.default_rng(31).random((29, 6))
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=500, n_reps=6, max_pts=500), shifts=sh)
    P1 = D.qmc_pnorm(Q)[0]
    Qd = D.QMCData_Distributions(Q)
    P2, _, _, r2 = D.qmc_pnorm(Qd, return_reps=True)
    F = Q.C
    _, _, _, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=500, n_reps=6, shifts=sh, cdf_form=1,
                                   gen_base0=0)
    np.testing.assert_allclose(r2, rc, rtol=1e-12)
    assert abs(P1 - P2) < 1e-12


def test_identity_known_answer_gpu(D):
    n = 20
    lo, up = W.bounds_quarter(np.eye(n))
    for prec, tol in ((L.PREC_FP64, 1e-14), (L.PREC_FP32_SIMT, 1e-6)):
        Q = D.QMCData(np.eye(n), lo, up, D.QMC_opts(m=512, n_reps=4), rng=np.random.default_rng(1),
                      precision=prec)
        P, err, _ = D.qmc_pnorm(Q)
        assert abs(P - 0.25) < tol


def test_equicorrelated_known_answer_gpu(D):
    n = 256
    S = W.fixed_dense(n)
    lo, up = W.bounds_quarter(S)
    ref = kat.equicorrelated(1.0, 1.0, lo, up)
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=4096, n_reps=12, max_pts=4096),
                  rng=np.random.default_rng(256))
    P, err, _ = D.qmc_pnorm(Q)
    assert abs(P - ref) < max(3 * err, 1e-3)


# ---------------------------------------------------------------- errors ---
def test_error_statuses(D):
    n = 6
    lo, up = -np.ones(n), np.ones(n)
    opts = D.QMC_opts(m=64, n_reps=2)
    B = np.random.default_rng(1).standard_normal((n, 2))
    with pytest.raises(D.DbgzError) as e:
        D.QMCData(B @ B.T, lo, up, opts)
    assert e.value.status == L.ERR_RANK_DEFICIENT
    S = np.eye(n)
    S[1, 2] = np.nan
    with pytest.raises(D.DbgzError) as e:
        D.QMCData(S, lo, up, opts)
    assert e.value.status == L.ERR_NONFINITE_INPUT
    S = np.eye(n)
    S[4, 4] = np.inf  # checked on the device, classic factor too
    with pytest.raises(D.DbgzError) as e:
        D.QMCDataSparse(S, lo, up, opts)
    assert e.value.status == L.ERR_NONFINITE_INPUT and "at 28" in str(e.value)
    with pytest.raises(D.DbgzError) as e:
        D.QMCData(np.eye(n), up, lo, opts)
    assert e.value.status == L.ERR_NONFINITE_INPUT
    with pytest.raises(D.DbgzError) as e:
        D.QMCData(np.eye(1), [-1.0], [1.0], opts)
    assert e.value.status == L.ERR_DIMENSION
    Q = D.QMCData(np.eye(n), lo, up, opts)
    with pytest.raises(D.DbgzError) as e:
        D.qmc_pnorm(Q, precision=17)
    assert e.value.status == L.ERR_INVALID_ARGUMENT


# ------------------------------------------------------- tensor-core loop ---
# FP32 numerics with the contraction on tcgen05: split BF16 (3 products) is
# held to the FP32-SIMT bar; TF32 (one product, 10-bit mantissa operands) to
# a looser one.
TC_TOL = {L.PREC_FP32_SPLIT_BF16: (5e-6, 2e-5), L.PREC_FP32_TF32: (1e-4, 2e-3)}


@pytest.mark.parametrize("prec", [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
@pytest.mark.parametrize("c", DENSE_CASES)
def test_pnorm_tensor_core_fixture(D, c, prec):
    z = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    g = _case(z, c)
    Q = _from_case(D, g, np.float32, precision=prec)
    P, err, npts, reps = D.qmc_pnorm(Q, return_reps=True)
    P64 = float(g["P"])
    at, rt = TC_TOL[prec]
    assert npts == int(g["n_pts"])
    assert abs(P - P64) <= at + rt * abs(P64), (P, P64, abs(P - P64))


@pytest.mark.parametrize("prec", [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
@pytest.mark.parametrize("n,m,n_reps", [(300, 777, 3), (600, 512, 2), (1000, 256, 2), (257, 300, 2)])
def test_pnorm_tensor_core_phases(D, n, m, n_reps, prec):
    # several 256-wide phases: the phase-start GEMM reads this tile's earlier
    # y's back from the workspace; partial tiles and a partial last block
    S = _spd(n, n + 7)
    lo, up = W.bounds_quarter(S)
    sh = np.random.default_rng(n).random((n - 1, n_reps))
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=m, n_reps=n_reps, max_pts=m, max_abs_err=0.0), shifts=sh)
    P64, _, _, r64 = D.qmc_pnorm(Q, precision=L.PREC_FP64, return_reps=True)
    Ps, _, _, rs = D.qmc_pnorm(Q, precision=L.PREC_FP32_SIMT, return_reps=True)
    Pt, _, _, rt_ = D.qmc_pnorm(Q, precision=prec, return_reps=True)
    at, rt = TC_TOL[prec]
    assert abs(Ps - P64) <= 5e-6 + 2e-5 * abs(P64), (Ps, P64)
    assert abs(Pt - P64) <= at + rt * abs(P64), (Pt, P64, abs(Pt - P64) / abs(P64))
    np.testing.assert_allclose(rt_, r64, rtol=10 * rt, atol=10 * at)


@pytest.mark.parametrize("prec", [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
@pytest.mark.parametrize("n,m,first", [(200, 1024, 2048), (600, 1024, 128 * 37), (300, 1000, 2048),
                                       (300, 1024, 2048 + 37), (300, 1000, None), (200, 1500, None)])
def test_pnorm_tensor_core_sobol_points(D, n, m, first, prec):
    # Sobol points in the tensor-core loop, from the per-block staged
    # integers at any first index: tiles at multiples of 128, at other
    # offsets, offsets that change from pass to pass (m not a multiple of 32),
    # and the default first index of SobolQMC (2^floor(log2(2m)) + 1); three
    # passes against the FP64 loop and the FP32 SIMT loop on the same points.
    # Other points would move P by about the QMC error, which the test
    # requires to be far above its tolerance.
    S = _spd(n, n + 11)
    lo, up = W.bounds_quarter(S)
    R = 3
    us = np.random.default_rng(n + m).integers(0, 2**64, size=(n - 1, R), dtype=np.uint64)
    opts = D.QMC_opts(m=m, n_reps=R, max_pts=3 * m, max_abs_err=0.0)
    out = {}
    for pr in (L.PREC_FP64, L.PREC_FP32_SIMT, prec):
        Q = D.QMCData(S, lo, up, opts, qmc_type="Sobol", ushifts=us, sobol_first=first)
        try:
            out[pr] = D.qmc_pnorm(Q, precision=pr, return_reps=True)
        finally:
            Q.close()
    P64, e64, n64, r64 = out[L.PREC_FP64]
    Ps, Pt, rt_ = out[L.PREC_FP32_SIMT][0], out[prec][0], out[prec][3]
    # same points: both precisions stay within 1e-6 here (d <= 600)
    tol = 5e-6 + 4e-5 * abs(P64)
    assert out[prec][2] == n64 == 3 * m
    assert e64 > 5 * tol, (e64, tol)
    assert abs(Pt - P64) <= tol and abs(Pt - Ps) <= tol, (Pt, Ps, P64)
    np.testing.assert_allclose(rt_, r64, rtol=0, atol=3 * tol)


@pytest.mark.parametrize("sparse", [False, True])
@pytest.mark.parametrize("m,first", [(1000, 2048), (1024, 128 * 19), (1000, 2085), (1000, None), (1500, None),
                                     (1024, None)])
def test_sobol_staged_points_fp64_vs_checker(D, oracle, sparse, m, first):
    # the FP64 loops (dense SIMT, banded) against the checker on Sobol points
    # from the per-block staged integers at any first index (partial last
    # tiles, offsets that change between passes, the default first index
    # 2^floor(log2(2m)) + 1 of SobolQMC for m a power of two and not)
    n, R = 160, 3
    S = _spd(n, 5 + m)
    lo, up = W.bounds_quarter(S)
    us = np.random.default_rng(m + (first or 0)).integers(0, 2**64, size=(n - 1, R), dtype=np.uint64)
    opts = D.QMC_opts(m=m, n_reps=R, max_pts=2 * m, max_abs_err=0.0)
    cls = D.QMCDataSparse if sparse else D.QMCData
    Q = cls(S, lo, up, opts, qmc_type="Sobol", ushifts=us, sobol_first=first)
    Q32 = cls(S, lo, up, opts, qmc_type="Sobol", ushifts=us, sobol_first=first)  # the same points again
    try:
        P, err, npts, reps = D.qmc_pnorm(Q, precision=L.PREC_FP64, return_reps=True)
        F = Q.C
        Pc, ec, nc, rc = oracle.qmc_pnorm(F.U, F.a, F.b, m=m, n_reps=R, max_pts=2 * m, max_abs_err=0.0,
                                          sparse=sparse, qmc_type=oracle.SOBOL, V=D.sobol_dirnums(n - 1),
                                          ushifts=us, sobol_first=Q.sobol_first)
        P32, _, _, r32 = D.qmc_pnorm(Q32, precision=L.PREC_FP32_SIMT, return_reps=True)
    finally:
        Q.close()
        Q32.close()
    assert npts == nc == 2 * m
    np.testing.assert_allclose(reps, rc, rtol=1e-12, atol=1e-300)
    assert ec > 5 * (5e-6 + 4e-5 * abs(Pc))  # other points would be seen below
    np.testing.assert_allclose(r32, rc, rtol=0, atol=5e-6 + 4e-5 * abs(Pc))


@pytest.mark.parametrize("prec", [L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
def test_identity_known_answer_tensor_core(D, prec):
    n = 40
    lo, up = W.bounds_quarter(np.eye(n))
    Q = D.QMCData(np.eye(n), lo, up, D.QMC_opts(m=1000, n_reps=4), rng=np.random.default_rng(2),
                  precision=prec)
    P, err, _ = D.qmc_pnorm(Q)
    assert abs(P - 0.25) < 1e-6


# ---------------------------------------------------------- sparse / banded ---
def test_pnorm_sparse_fixture(D):
    z = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    g = _case(z, "tridiag8")
    Q = _from_case(D, g)
    P, err, npts, reps = D.qmc_pnorm(Q, return_reps=True)
    assert npts == int(g["n_pts"])
    np.testing.assert_allclose(reps, g["reps"], rtol=1e-12, atol=1e-300)
    Q32 = _from_case(D, g, np.float32, precision=L.PREC_FP32_SIMT)
    P32 = D.qmc_pnorm(Q32)[0]
    assert abs(P32 - float(g["P"])) <= 2e-6 + 1e-5 * abs(float(g["P"]))


def _ar1(n, rho=0.9):
    i = np.arange(n)
    return rho ** np.abs(i[:, None] - i[None, :])


def _blocks(sizes, seed):
    # block-diagonal SPD with irregular blocks: the classic factor keeps the
    # blocks, so its CSC has columns of every length from 0 up (a general
    # sparsity pattern, not a band)
    rng = np.random.default_rng(seed)
    n = sum(sizes)
    S = np.zeros((n, n))
    o = 0
    for k in sizes:
        A = rng.standard_normal((k, k + 3))
        S[o:o + k, o:o + k] = W.correlation(A @ A.T)
        o += k
    return S


@pytest.mark.parametrize("n,band,qmc", [(60, None, "Richtmyer"), (300, 16, "Richtmyer"),
                                         (300, 64, "Sobol"), (600, None, "Richtmyer"),
                                         (120, "blocks", "Sobol")])
def test_pnorm_sparse_vs_checker(D, oracle, n, band, qmc):
    # classic factor, CSC of the strict upper triangle (optionally band-limited);
    # n = 600 without a band exceeds the shared-memory ring (global ring path)
    blocks = band == "blocks"
    if blocks:
        band = None
    S = _blocks([5, 17, 1, 40, 9, 48], 7) if blocks else (_spd(n, n) if band is None else _ar1(n))
    rng = np.random.default_rng(n + 1)
    if blocks:
        assert np.count_nonzero(np.triu(S, 1)) < n * (n - 1) // 4
    a = np.full(n, -np.inf) if band else W.bounds_quarter(S)[0]
    b = rng.uniform(-0.5, 2.5, n) if band else W.bounds_quarter(S)[1]
    m, n_reps = 500, 3
    kw = {}
    if qmc == "Richtmyer":
        kw["shifts"] = rng.random((n - 1, n_reps))
    else:
        kw["ushifts"] = rng.integers(0, 2**64, size=(n - 1, n_reps), dtype=np.uint64)
    Q = D.QMCDataSparse(S, a, b, D.QMC_opts(m=m, n_reps=n_reps, max_pts=m, max_abs_err=0.0), qmc_type=qmc, **kw)
    if band:
        Q.truncate_band(band)
    F = Q.C
    U = F.U.copy()
    if band:
        assert np.all(np.triu(U, band + 1) == 0)
    if blocks:
        assert np.all(U[S == 0] == 0)  # the factor keeps the block pattern
    P, err, npts, reps = D.qmc_pnorm(Q, precision=L.PREC_FP64, return_reps=True)
    okw = dict(m=m, n_reps=n_reps, sparse=True, max_pts=m)
    if qmc == "Richtmyer":
        okw["shifts"] = kw["shifts"]
    else:
        okw.update(qmc_type=oracle.SOBOL, V=D.sobol_dirnums(n - 1), ushifts=kw["ushifts"], sobol_first=Q.sobol_first)
    Pc, ec, nc, rc = oracle.qmc_pnorm(U, F.a, F.b, **okw)
    np.testing.assert_allclose(reps, rc, rtol=1e-12, atol=1e-300)
    P32, _, _, r32 = D.qmc_pnorm(Q, precision=L.PREC_FP32_SIMT, return_reps=True)
    assert abs(P32 - Pc) <= 5e-6 + 2e-5 * abs(Pc), (P32, Pc)


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_FP32_SIMT, L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32])
@pytest.mark.parametrize("gen,sparse", [("Richtmyer", False), ("Sobol", False), ("Sobol", True)])
def test_one_sided_step_same_bits(D, prec, gen, sparse):
    # with every lower bound -inf the loops take the one-sided step (the lower
    # CDF value is one constant); a = -1e300 takes the general step through
    # the same clamped argument: the per-shift means must be the same bits
    if sparse and prec in (L.PREC_FP32_SPLIT_BF16, L.PREC_FP32_TF32):
        pytest.skip("the banded loop has no tensor-core modes")
    n, m, R = 150, 1000, 3
    S = _spd(n, 17)
    rng = np.random.default_rng(18)
    b = rng.uniform(-1.0, 2.5, n)
    opts = D.QMC_opts(m=m, n_reps=R, max_pts=2 * m, max_abs_err=0.0)
    kw = dict(shifts=rng.random((n - 1, R))) if gen == "Richtmyer" else \
        dict(qmc_type="Sobol", ushifts=rng.integers(0, 2**64, size=(n - 1, R), dtype=np.uint64))
    cls = D.QMCDataSparse if sparse else D.QMCData
    out = []
    for lo in (-np.inf, -1e300):
        Q = cls(S, np.full(n, lo), b, opts, **kw)
        try:
            out.append(D.qmc_pnorm(Q, precision=prec, return_reps=True))
        finally:
            Q.close()
    assert out[0][2] == out[1][2] == 2 * m
    assert np.array_equal(out[0][3], out[1][3]) and out[0][0] == out[1][0]

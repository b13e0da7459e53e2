"""The CPU checker pinned against the reference's own assertions, its known
answers and its published values (no GPU).  Each test cites the reference
test or data it restates."""
import json
import math
import os

import numpy as np
import pytest
from scipy.special import erfinv as sp_erfinv

from dbgenzpaper_b200 import workloads as W
from oracle import kat

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_det_erf_exp_accuracy(oracle):
    for x in np.linspace(-7, 7, 1401):
        r = math.erf(x)
        v = oracle.det_erf(x)
        assert abs(v - r) <= 5 * math.ulp(r if r != 0 else 1e-300) or v == r
    for x in np.linspace(-700, 700, 1401):
        r = math.exp(x)
        assert abs(oracle.det_exp(x) - r) <= math.ulp(r)
    assert oracle.det_erf(float("inf")) == 1.0 and oracle.det_erf(-float("inf")) == -1.0
    assert math.isnan(oracle.det_erf(float("nan")))
    assert oracle.det_exp(-float("inf")) == 0.0


def test_det_erf_within_two_ulp_of_correctly_rounded(oracle):
    # the fitted polynomials of det_erf against 40-digit erf rounded once
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 40
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(0, 6.5, 3000), rng.uniform(0, 1e-3, 200),
                         2.5 * (1 + rng.uniform(-1e-9, 1e-9, 200)), -rng.uniform(0, 6.5, 200)])
    for x in xs:
        r = float(mp.erf(mp.mpf(float(x))))
        assert abs(oracle.det_erf(float(x)) - r) <= 2 * math.ulp(r if r != 0 else 1e-300), x


def test_det_erf_tables_match_their_fit():
    # the coefficient tables in detmath.h are what detmath_fit.py prints
    import contextlib
    import importlib.util
    import io
    import re
    here = os.path.join(os.path.dirname(os.path.dirname(__file__)), "dbgenzpaper_b200", "csrc")
    pytest.importorskip("mpmath")
    spec = importlib.util.spec_from_file_location("detmath_fit", os.path.join(here, "detmath_fit.py"))
    fit = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(fit)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        fit.main()
    header = open(os.path.join(here, "detmath.h")).read()

    def table(text, name):
        body = re.search(r"#define %s \{(.*?)\}" % name, text, re.S).group(1)
        return [float.fromhex(v.strip()) for v in body.replace("\\", "").split(",")]

    for name in ("DBGZ_ERF_SMALL_TABLE", "DBGZ_ERFC_MID_TABLE"):
        assert table(header, name) == table(buf.getvalue(), name)


def test_erfinv_accuracy(oracle):
    for u in np.concatenate([np.linspace(-0.999999, 0.999999, 801), [1 - 2e-16, -1 + 2e-16, 1e-300]]):
        r = sp_erfinv(u)
        assert abs(oracle.erfinv(u) - r) <= 4e-16 * abs(r) + 1e-300


def test_cholesky_genz_reconstruction(oracle):
    # test/runtests.jl:15-36 (n = 1024, A ~ U(0,1), C = A A' + 100 I)
    rng = np.random.default_rng(101)
    n = 1024
    A = rng.random((n, n))
    C = A @ A.T + 100.0 * np.eye(n)
    F = oracle.cholesky_genz(C, -np.ones(n), np.ones(n))
    U = np.triu(F["U"])
    p = F["perm"]
    d = np.sqrt(np.diag(C))
    Ct = C / np.outer(d, d)
    assert F["rank"] == n
    assert sorted(p) == list(range(n))
    assert np.max(np.abs(Ct[np.ix_(p, p)] - U.T @ U)) < 1e-10


def test_cholesky_genz_reorders_by_probability(oracle):
    # with Sigma = I the Genz order is ascending marginal probability mass
    n = 12
    rng = np.random.default_rng(5)
    b = rng.uniform(0.1, 3.0, n)
    F = oracle.cholesky_genz(np.eye(n), -np.full(n, np.inf), b, 4, 6)
    for p0 in (0, 6):  # panel-restricted pivoting (bs2 = 6)
        panel = F["perm"][p0:p0 + 6]
        assert list(panel) == list(np.sort(np.arange(p0, p0 + 6))[np.argsort(b[p0:p0 + 6], kind="stable")])


@pytest.mark.parametrize("bs", [8, 16, 32, 64])
def test_cholesky_classic_reconstruction(oracle, bs):
    # test/runtests.jl:38-59
    rng = np.random.default_rng(102)
    n = 100
    A = rng.random((n, n))
    C = A @ A.T + 100.0 * np.eye(n)
    d = np.sqrt(np.diag(C))
    Ct = C / np.outer(d, d)
    F = oracle.cholesky_classic(C, -np.ones(n), np.ones(n), bs, bs, bs, bs)
    U = np.triu(F["U"])
    assert np.max(np.abs(Ct - U.T @ U)) < 1e-10


def test_richtmyer_properties(oracle):
    # test/runtests.jl:91-113
    n_dim, n_pts = 1024, 1024
    q = oracle.sqrt_primes(n_dim)
    assert q.dtype == np.float64 and np.all((0 < q) & (q < 1))
    X = oracle.richtmyer_mat(n_pts, q, 0)
    assert len(np.unique(X[:, -1].astype(np.float32))) == n_pts
    X2 = oracle.richtmyer_mat(n_pts, q, n_pts)
    assert len(np.unique(X2[:, -1].astype(np.float32))) == n_pts
    X3 = oracle.richtmyer_mat(n_pts, q, 2**20)
    assert len(np.unique(X3[:, -1].astype(np.float32))) == n_pts
    # X[i, j] = frac((n0 + i) q_j) exactly
    i = np.arange(1, n_pts + 1, dtype=np.float64)
    assert np.array_equal(X[:, 3], i * q[3] - np.floor(i * q[3]))


def test_sobol_net_property(oracle):
    import ctypes as C
    from dbgenzpaper_b200 import _lib as L
    dims = 50
    V = np.zeros((dims, 32), dtype=np.uint32)
    L.check(L.lib().dbgz_sobol_dirnums(dims, V.ctypes.data_as(C.POINTER(C.c_uint32))))
    k = 10
    X = oracle.sobol_points(V, 3 * 2**k, 2**k)  # an aligned block of 2^k points
    for j in range(dims):
        assert len(np.unique(X[:, j] >> (32 - k))) == 2**k
    # first points of the van der Corput dimension
    X0 = oracle.sobol_points(V[:1], 1, 4)[:, 0] / 2.0**32
    assert list(X0) == [0.5, 0.75, 0.25, 0.375]


def _prep(oracle, S, a, b, bs=(64, 512), sparse=False):
    F = (oracle.cholesky_classic if sparse else oracle.cholesky_genz)(S, a, b, *bs)
    return oracle.truncate_U(F["U"]), F


def test_identity_known_answer(oracle):
    n = 16
    lo, up = W.bounds_quarter(np.eye(n))
    U, F = _prep(oracle, np.eye(n), lo, up)
    sh = np.random.default_rng(1).random((n - 1, 12))
    P, err, npts, reps = oracle.qmc_pnorm(U, F["a"], F["b"], m=256, n_reps=12, shifts=sh)
    assert abs(P - 0.25) < 1e-14 and err < 1e-13 and npts == 256


def test_dense_vs_independent_integrator(oracle):
    # test/runtests.jl:150-173 (MvNormalCDF replaced by scipy's Genz-Bretz)
    rng = np.random.default_rng(42)
    n = 8
    S = W.rand_spd(n, 4.0, rng)
    a, b = np.full(n, -np.inf), np.full(n, 2.0)
    U, F = _prep(oracle, S, a, b)
    sh = rng.random((n - 1, 12))
    P, err, npts, _ = oracle.qmc_pnorm(U, F["a"], F["b"], m=2**11, n_reps=12, shifts=sh,
                                       block_size_i=256, block_size_i2=64, block_size_j=128,
                                       max_pts=2**13, max_abs_err=0.0)
    ref = kat.scipy_mvn(S, a, b)
    assert np.isfinite(P) and np.isfinite(err) and npts == 2**13
    assert abs(P - ref) < 0.06           # the reference test's tolerance
    assert abs(P - ref) < 3 * err + 1e-6  # and the QMC error bound


def test_sparse_vs_independent_integrator(oracle):
    # test/runtests.jl:175-201 (tridiagonal 1.8 / 0.25, b = 1.5)
    n = 8
    S = np.diag(np.full(n, 1.8)) + np.diag(np.full(n - 1, 0.25), 1) + np.diag(np.full(n - 1, 0.25), -1)
    a, b = np.full(n, -np.inf), np.full(n, 1.5)
    U, F = _prep(oracle, S, a, b, sparse=True)
    sh = np.random.default_rng(21).random((n - 1, 12))
    P, err, npts, _ = oracle.qmc_pnorm(U, F["a"], F["b"], m=2**11, n_reps=12, shifts=sh,
                                       sparse=True, max_pts=2**13, max_abs_err=0.0)
    ref = kat.scipy_mvn(S, a, b)
    assert abs(P - ref) < 0.06 and abs(P - ref) < 3 * err + 1e-6


def test_equicorrelated_published_value(oracle):
    # Sigma_2 = 1 1' + I at n = 256: closed form (mwp.jl:80-116) against the
    # reference's published estimate (data/sims/table_sparse_dense1.tex:10)
    pub = json.load(open(os.path.join(GOLD, "published.json")))
    row = pub["rows"][0]
    n = row["n"]
    S = W.fixed_dense(n)
    lo, up = W.bounds_quarter(S)
    assert abs(row["closed_form"] - kat.equicorrelated(1.0, 1.0, lo, up)) < 1e-12
    for r in pub["rows"]:
        assert abs(r["value"] - r["closed_form"]) < 3 * r["sd"] + 1e-4
    U, F = _prep(oracle, S, lo, up)
    sh = np.random.default_rng(256).random((n - 1, 12))
    P, err, _, _ = oracle.qmc_pnorm(U, F["a"], F["b"], m=1024, n_reps=12, shifts=sh)
    assert abs(P - row["closed_form"]) < max(3 * err, 3 * row["sd"])


def test_distributions_variant_agrees(oracle):
    # erf form vs erfc form on the same points (simulation_precision.jl:94-123)
    S = W.rand_spd(30, 1.0, np.random.default_rng(30))
    lo, up = W.bounds_quarter(S)
    U, F = _prep(oracle, S, lo, up)
    sh = np.random.default_rng(3).random((29, 12))
    P1 = oracle.qmc_pnorm(U, F["a"], F["b"], m=512, n_reps=12, shifts=sh, cdf_form=0)[0]
    P2 = oracle.qmc_pnorm(U, F["a"], F["b"], m=512, n_reps=12, shifts=sh, cdf_form=1)[0]
    assert abs(P1 - P2) < 1e-13


def test_golden_fixtures_reproduce(oracle):
    z = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    names = sorted({k.split("/")[0] for k in z.files})
    assert {"c1", "spd8", "sobol40", "tridiag8", "erfc130"} <= set(names)
    for c in names:
        g = lambda k: z[f"{c}/{k}"]
        sparse = bool(g("sparse"))
        U, F = _prep(oracle, g("Sigma"), g("a_in"), g("b_in"), (int(g("bs1")), int(g("bs2"))), sparse)
        assert np.array_equal(U, g("U"), equal_nan=True) and np.array_equal(F["perm"], g("perm"))
        kw = dict(m=int(g("m")), n_reps=int(g("n_reps")), max_pts=int(g("max_pts")), max_abs_err=0.0,
                  cdf_form=int(g("cdf_form")), sparse=sparse)
        if int(g("qmc_type")) == 0:
            kw["shifts"] = g("shifts")
        else:
            kw.update(qmc_type=1, V=g("V"), ushifts=g("ushifts"), sobol_first=int(g("sobol_first")))
        P, err, npts, reps = oracle.qmc_pnorm(U, F["a"], F["b"], **kw)
        assert np.array_equal(reps, g("reps")) and P == float(g("P")) and npts == int(g("n_pts"))


def test_continuation_matches_longer_run(oracle):
    # a pass that starts at generator offset m equals the second pass of a
    # two-pass run (next_points!, src/qmc_generators.jl:119-122)
    S = W.rand_spd(12, 2.0, np.random.default_rng(12))
    lo, up = W.bounds_quarter(S)
    U, F = _prep(oracle, S, lo, up)
    sh = np.random.default_rng(4).random((11, 4))
    _, _, _, r2 = oracle.qmc_pnorm(U, F["a"], F["b"], m=300, n_reps=4, shifts=sh, max_pts=600,
                                   max_abs_err=0.0)
    _, _, _, r1 = oracle.qmc_pnorm(U, F["a"], F["b"], m=300, n_reps=4, shifts=sh)
    _, _, _, rb = oracle.qmc_pnorm(U, F["a"], F["b"], m=300, n_reps=4, shifts=sh, gen_base0=300)
    assert np.allclose(r2, 0.5 * (r1 + rb), rtol=1e-14, atol=0)


def test_pivot_margins_log(oracle):
    # ties (equicorrelated, equal bounds) log a zero margin and keep the
    # lowest index; the log changes nothing in the factorisation
    n = 8
    S = 0.5 * np.ones((n, n)) + 0.5 * np.eye(n)
    F = oracle.cholesky_genz(S, -np.ones(n), np.ones(n), margins=True)
    assert np.array_equal(F["perm"], np.arange(n))
    assert np.all(F["margins"][:-1] == 0.0) and np.isinf(F["margins"][-1])
    rng = np.random.default_rng(3)
    A = rng.standard_normal((30, 40))
    S = A @ A.T
    lo, up = -rng.uniform(0.5, 2, 30), rng.uniform(0.5, 2, 30)
    F1 = oracle.cholesky_genz(S, lo, up, margins=True)
    F2 = oracle.cholesky_genz(S, lo, up)
    assert np.array_equal(F1["U"], F2["U"]) and np.array_equal(F1["perm"], F2["perm"])
    assert np.all(F1["margins"][np.isfinite(F1["margins"])] >= 0.0)


# ---- the timed CPU baseline (oracle/genz_cpu_blas.c) against the checker --
@pytest.mark.parametrize("isa", ["avx2", "avx512"])
def test_cpu_blas_pass_matches_checker(oracle, isa, monkeypatch):
    """The BLAS-3, vectorised restatement of qmc_loop! that bench.py times
    (src/qmc.jl:315-444) gives the checker's per-shift means to 1e-13
    relative: both generators, partial last tiles, tile heights that are not
    multiples of 8, several outer and inner dimension blocks."""
    if isa == "avx512" and oracle.cpu_isa() != "avx512":
        pytest.skip("no AVX-512 on this CPU")
    monkeypatch.setattr(oracle, "_cpu", None)
    monkeypatch.setattr(oracle, "cpu_isa", lambda: isa)
    from oracle.oracle import sqrt_primes  # noqa: F401  (the checker is built)
    rng = np.random.default_rng(77)
    for d, m, bj, bi, bi2 in ((33, 500, 20, 16, 8), (150, 777, 100, 64, 32), (301, 300, 64, 128, 32)):
        S = W.rand_spd(d, 1.0, rng)
        lo, up = W.bounds_quarter(S)
        F = oracle.cholesky_genz(S, lo, up)
        U = oracle.truncate_U(F["U"])
        sh = rng.random((d - 1, 3))
        r_fast = oracle.qmc_pass_blas(U, F["a"], F["b"], m=m, n_reps=3, shifts=sh, block_size_j=bj,
                                      block_size_i=bi, block_size_i2=bi2, threads=2)
        r_chk = oracle.qmc_pnorm(U, F["a"], F["b"], m=m, n_reps=3, shifts=sh)[3]
        np.testing.assert_allclose(r_fast, r_chk, rtol=1e-13, atol=0)
        V = W.sobol_table(d - 1) if hasattr(W, "sobol_table") else None
        if V is None:
            import dbgenzpaper_b200 as D
            V = D.sobol_dirnums(d - 1)
        us = rng.integers(0, 2**63, size=(d - 1, 3), dtype=np.uint64)
        first = 2 * m + 1
        r_fast = oracle.qmc_pass_blas(U, F["a"], F["b"], m=m, n_reps=3, qmc_type=oracle.SOBOL, V=V,
                                      ushifts=us, sobol_first=first, block_size_j=bj, block_size_i=bi,
                                      block_size_i2=bi2, threads=2)
        r_chk = oracle.qmc_pnorm(U, F["a"], F["b"], m=m, n_reps=3, qmc_type=oracle.SOBOL, V=V, ushifts=us,
                                 sobol_first=first)[3]
        np.testing.assert_allclose(r_fast, r_chk, rtol=1e-13, atol=0)


def test_cpu_blas_erfinv(oracle):
    """The vectorised erfinv of the CPU baseline against the checker's
    Newton-refined one: relative error < 1e-13 where |x| >= 1e-3, absolute
    < 1e-15 everywhere (the Halley step works on erfc(x) = 1 - |x|, so near
    0 the error is absolute, about 1e-17)."""
    x = np.concatenate([np.linspace(-1 + 4.4e-16, 1 - 4.4e-16, 20001), 1 - np.logspace(-15.6, -0.3, 500),
                        -1 + np.logspace(-15.6, -0.3, 500), np.logspace(-12, -1, 200)])
    y = oracle.cpu_erfinv(x)
    yo = np.array([oracle.erfinv(v) for v in x])
    big = np.abs(x) >= 1e-3
    assert np.max(np.abs(y[big] - yo[big]) / np.abs(yo[big])) < 1e-13
    assert np.max(np.abs(y - yo)) < 1e-15


# ---- cholesky_rowmax! and adapt_low_rank! (src/cholesky.jl:24-123, 244-432)
def test_adapt_low_rank_reference_testset(oracle):
    """test/runtests.jl:61-89: a rank-20 factor with 10 dependent columns,
    column 25 (1-based) all zero: one zero-level column, moved to the end."""
    rng = np.random.default_rng(61)
    n, rank = 30, 20
    M = np.zeros((n, n))
    M[np.arange(rank), np.arange(rank)] = 1.0
    M[:rank, rank:] = rng.random((rank, n - rank))
    M[:, 24] = 0.0
    a, b = np.zeros(n), np.ones(n)
    M2, a2, b2, perm, k_js, k_0 = oracle.adapt_low_rank(M, a, b, rank, np.arange(n), 1e-10)
    assert k_0 == 1
    assert perm[-1] == 24
    assert np.all(M2[:, -1] == 0.0)
    assert len(k_js) == rank
    # every column is where its level puts it, scaled so its last entry is 1
    assert sorted(perm.tolist()) == list(range(n))
    assert k_js[-1] == n - k_0


def test_adapt_low_rank_levels_and_signs(oracle):
    """Columns of every level, negative pivots (bounds swapped), several
    zero columns: the block structure k_js, the scaling and the order."""
    rng = np.random.default_rng(62)
    n, rank = 40, 12
    M = np.zeros((n, n))
    M[np.arange(rank), np.arange(rank)] = 1.0
    lev = rng.integers(0, rank + 1, size=n - rank)  # 0: a zero column
    for c, l in zip(range(rank, n), lev):
        if l:
            M[:l, c] = rng.standard_normal(l)
            M[l - 1, c] = rng.choice([-1.0, 1.0]) * (0.5 + rng.random())
    a, b = -rng.random(n), rng.random(n)
    M2, a2, b2, perm, k_js, k_0 = oracle.adapt_low_rank(M, a, b, rank, np.arange(n), 1e-12)
    assert k_0 == int(np.sum(lev == 0))
    for t in range(n - k_0):
        c = perm[t]
        if c >= rank:
            l = lev[c - rank]
            m = M[l - 1, c]
            assert np.array_equal(M2[:l, t], M[:l, c] * (1.0 / m))
            lo, hi = a[c] * (1.0 / m), b[c] * (1.0 / m)
            assert (a2[t], b2[t]) == ((hi, lo) if m < 0 else (lo, hi))
    # blocks: level-i constraints sit right after base column i-1 and its earlier ones
    starts = [0] + list(k_js[:-1])
    for i in range(rank):
        assert perm[starts[i]] == i
        for t in range(starts[i] + 1, k_js[i]):
            assert lev[perm[t] - rank] == i + 1


@pytest.mark.parametrize("n,rank_true,bs", [(60, 60, (8, 16, 32, 64)), (100, 37, (16, 32, 64, 128)),
                                            (300, 300, (64, 128, 256, 512))])
def test_cholesky_rowmax_reconstruction(oracle, n, rank_true, bs):
    """Diagonal pivoting: the permuted correlation matrix is U'U to 1e-10
    (the bound of test/runtests.jl:15-36) on the leading rank block, the
    pivots take the largest remaining diagonal, and a rank-deficient matrix
    stops at its rank."""
    rng = np.random.default_rng(n + rank_true)
    A = rng.standard_normal((n, rank_true))
    S = A @ A.T + (0.0 if rank_true < n else 0.5) * np.eye(n)
    a, b = -np.ones(n), np.ones(n)
    F = oracle.cholesky_rowmax(S, a, b, *bs)
    d = np.sqrt(np.diag(S))
    R = S / np.outer(d, d)
    p = F["perm"]
    r = F["rank"]
    # the rank test is m_ii > 0 (src/cholesky.jl:309-314), not against a
    # tolerance: past the true rank the pivots are rounding residue (about
    # 1e-8 after the square root) until one is not positive
    assert (r == n) if rank_true == n else (rank_true <= r < n)
    if rank_true < n:
        assert np.all(np.diag(F["U"])[rank_true:r] < 1e-6)
    r = rank_true
    U = np.triu(F["U"])[:r, :r]
    assert np.max(np.abs(R[np.ix_(p[:r], p[:r])] - U.T @ U)) < 1e-10
    # a and b are scaled in place but not permuted (src/cholesky.jl:265-266)
    np.testing.assert_array_equal(F["a"], a / d)

"""cholesky_rowmax! and adapt_low_rank! on the GPU against the checker
(needs a B200): the factor, permutation, rank and bounds bit for bit, and the
reference's own adapt_low_rank! testset (test/runtests.jl:61-89)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def D(dbgz):
    dbgz.get_context(0)
    return dbgz


@pytest.mark.parametrize("n,rank_true,bs", [(7, 7, (64, 512, 1024, 2048)), (130, 130, (16, 64, 1024, 2048)),
                                            (300, 300, (64, 128, 256, 512)), (100, 37, (16, 32, 64, 128)),
                                            (600, 600, (128, 512, 1024, 2048))])
def test_cholesky_rowmax_bitexact(D, oracle, n, rank_true, bs):
    rng = np.random.default_rng(n * 7 + rank_true)
    A = rng.standard_normal((n, rank_true))
    S = A @ A.T + (0.0 if rank_true < n else 0.5) * np.eye(n)
    a, b = rng.uniform(-3, 0, n), rng.uniform(0, 3, n)
    G = D.cholesky_rowmax(S, a, b, *bs)
    F = oracle.cholesky_rowmax(S, a, b, *bs)
    assert G.rank == F["rank"]
    assert np.array_equal(G.perm, F["perm"])
    assert np.array_equal(G.U, F["U"])
    assert np.array_equal(G.a, F["a"]) and np.array_equal(G.b, F["b"])
    assert np.array_equal(G.scale_vec, F["scale_vec"])


def test_cholesky_rowmax_ties_take_the_first(D, oracle):
    # the identity: every remaining diagonal ties at 1, so no pivot moves
    n = 70
    G = D.cholesky_rowmax(np.eye(n), -np.ones(n), np.ones(n), 16, 32)
    assert G.rank == n and np.array_equal(G.perm, np.arange(n))


def test_adapt_low_rank_reference_testset(D, oracle):
    rng = np.random.default_rng(61)
    n, rank = 30, 20
    M = np.zeros((n, n))
    M[np.arange(rank), np.arange(rank)] = 1.0
    M[:rank, rank:] = rng.random((rank, n - rank))
    M[:, 24] = 0.0
    out = D.adapt_low_rank(M, np.zeros(n), np.ones(n), rank, np.arange(n), 1e-10)
    M2, a2, b2, perm, k_js, k_0 = out
    assert k_0 == 1 and perm[-1] == 24 and np.all(M2[:, -1] == 0.0) and len(k_js) == rank
    ref = oracle.adapt_low_rank(M, np.zeros(n), np.ones(n), rank, np.arange(n), 1e-10)
    for x, y in zip(out, ref):
        assert np.array_equal(np.asarray(x), np.asarray(y))


@pytest.mark.parametrize("n,rank,nr", [(40, 12, 40), (300, 100, 300), (64, 64, 64), (50, 0, 50), (33, 10, 12)])
def test_adapt_low_rank_matches_checker(D, oracle, n, rank, nr):
    rng = np.random.default_rng(n + rank)
    M = np.zeros((nr, n))
    M[np.arange(rank), np.arange(rank)] = 1.0
    lev = rng.integers(0, rank + 1, size=n - rank)
    for c, lv in zip(range(rank, n), lev):
        if lv:
            M[:lv, c] = rng.standard_normal(lv)
            M[lv - 1, c] = rng.choice([-1.0, 1.0]) * (0.5 + rng.random())
            if lv < rank:
                M[lv:rank, c] = 1e-13 * rng.standard_normal(rank - lv)  # below eps1: not part of the level
    M[rank:, :] += rng.standard_normal((nr - rank, n)) if nr > rank else 0.0
    a, b = -rng.random(n), rng.random(n)
    perm = rng.permutation(n)
    got = D.adapt_low_rank(M, a, b, rank, perm, 1e-10)
    ref = oracle.adapt_low_rank(M, a, b, rank, perm, 1e-10)
    for x, y in zip(got, ref):
        assert np.array_equal(np.asarray(x), np.asarray(y))

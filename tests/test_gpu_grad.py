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
@pytest.mark.parametrize("n", [50, 300])
def test_fp32_gradients_close_to_fp64(dbgz, prec, tol, n):
    # n = 300 crosses the tensor loop's 256-wide phases in both directions
    D = dbgz
    Q = _problem(D, n, 2000 + n)
    P64, _, _, da64, db64, dU64 = D.qmc_pnorm_grad(Q, precision=L.PREC_FP64)
    P, _, _, da, db, dU = D.qmc_pnorm_grad(Q, precision=prec)
    assert abs(P - P64) <= 1e-4 * abs(P64) + 1e-6
    for g, g64 in ((da, da64), (db, db64), (dU, dU64)):
        assert np.linalg.norm(g - g64) <= tol * np.linalg.norm(g64), (np.linalg.norm(g - g64) / np.linalg.norm(g64))

"""Known-answer probabilities for checking the integrators (test infrastructure).

* ``equicorrelated(alpha, beta, lower, upper)`` -- P(lower <= X <= upper) for
  X ~ N(0, alpha I + beta 1 1'), restating the reference's own known answer
  (scripts/simulations/mwp.jl:80-116, temp.jl:40-76): conditioning on the
  common factor Z reduces the d-dimensional probability to a 1-D expectation
  E_Z[prod_i (Phi((u_i - sqrt(beta) Z)/sqrt(alpha)) - Phi((l_i - ...)/...))],
  evaluated with the trapezoid rule on z in [-12, 12] (exponentially
  convergent for this smooth, Gaussian-weighted integrand), product in logs.
* ``independent(lower, upper)`` -- prod_i (Phi(u_i) - Phi(l_i)) for Sigma = I.
* ``scipy_mvn(Sigma, lower, upper)`` -- scipy's Genz-Bretz integrator, an
  independent implementation used in place of the Julia package MvNormalCDF
  the reference tests compare against (test/runtests.jl:150-201).
"""
from __future__ import annotations

import numpy as np
from scipy.special import log_ndtr, ndtr


def _log_diff_cdf(u, l):
    # log(Phi(u) - Phi(l)) for u > l, stable in both tails
    lu, ll = log_ndtr(u), log_ndtr(l)
    lu2, ll2 = log_ndtr(-l), log_ndtr(-u)  # upper-tail form
    with np.errstate(divide="ignore", invalid="ignore"):
        lower_form = lu + np.log1p(-np.exp(ll - lu))
        upper_form = lu2 + np.log1p(-np.exp(ll2 - lu2))
    return np.where(l > 0, upper_form, lower_form)


def equicorrelated(alpha: float, beta: float, lower, upper, nodes: int = 6001) -> float:
    lower = np.asarray(lower, dtype=np.float64)
    upper = np.asarray(upper, dtype=np.float64)
    z = np.linspace(-12.0, 12.0, nodes)
    w = np.full(nodes, z[1] - z[0]) * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)
    w[0] *= 0.5
    w[-1] *= 0.5
    sa, sb = np.sqrt(alpha), np.sqrt(beta)
    shift = sb * z[:, None]
    lp = _log_diff_cdf((upper[None, :] - shift) / sa, (lower[None, :] - shift) / sa).sum(axis=1)
    return float(np.sum(w * np.exp(lp)))


def independent(lower, upper) -> float:
    return float(np.prod(ndtr(np.asarray(upper)) - ndtr(np.asarray(lower))))


def scipy_mvn(Sigma, lower, upper, seed: int = 7, maxpts: int = 2_000_000, abseps: float = 1e-7):
    from scipy.stats import multivariate_normal
    n = Sigma.shape[0]
    mvn = multivariate_normal(mean=np.zeros(n), cov=Sigma, allow_singular=False,
                              maxpts=maxpts, abseps=abseps, releps=0, seed=seed)
    return float(mvn.cdf(np.asarray(upper), lower_limit=np.asarray(lower)))

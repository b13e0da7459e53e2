"""Seeded synthetic workloads.

The reference's experiments draw their inputs from Julia's global RNG
(scripts/simulations/simulations_functions.jl); the generators below
produce inputs of the same families, shapes and value distributions from
numpy's PCG64 with fixed seeds, so every implementation (GPU kernels, CPU
checker, reference-arm baseline) sees the same Sigma, bounds and shifts.

Families of the reference (simulations_functions.jl:13-79):
  rand_spd(n; jitter)  A A' + jitter n I, A ~ N(0,1) n x n
  fixed_dense(n)       1 1' + I   (the paper's Sigma_2)
  fixed_sparse(n, k)   banded, diag k/2*2, ones on k off-diagonals
  bounds_quarter(S)    +-k sqrt(S_ii), k = Phi^-1((1 + 0.25^(1/n))/2),
                       so that the independent case has P = 0.25
Benchmark configurations (c1 .. c5) of the Genz path at d = 10 .. 10^4.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np
from scipy.special import ndtri


def correlation(S: np.ndarray) -> np.ndarray:
    d = np.sqrt(np.diag(S))
    R = S / np.outer(d, d)
    np.fill_diagonal(R, 1.0)
    return (R + R.T) / 2


def rand_spd(n: int, jitter: float = 1.0, rng=None) -> np.ndarray:
    rng = np.random.default_rng(0) if rng is None else rng
    A = rng.standard_normal((n, n))
    S = A @ A.T + jitter * n * np.eye(n)
    return (S + S.T) / 2


def fixed_dense(n: int, jitter: float = 1.0) -> np.ndarray:
    return np.ones((n, n)) + jitter * np.eye(n)


def fixed_sparse(n: int, n_sp: int) -> np.ndarray:
    M = np.diag(np.full(n, n_sp / 2.0))
    for i in range(1, n_sp + 1):
        M += np.diag(np.ones(n - i), i)
    return M + M.T


def bounds_quarter(S: np.ndarray):
    n = S.shape[0]
    k = ndtri((1 + 0.25 ** (1 / n)) / 2)
    s = np.sqrt(np.diag(S))
    return -s * k, s * k


@dataclass
class Workload:
    name: str
    Sigma: np.ndarray
    a: np.ndarray
    b: np.ndarray
    qmc_type: str          # "Richtmyer" | "Sobol"
    m: int                 # points per shift
    n_reps: int            # shifts
    shifts: Optional[np.ndarray] = None   # Richtmyer (d-1) x n_reps
    ushifts: Optional[np.ndarray] = None  # Sobol (d-1) x n_reps
    note: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def d(self) -> int:
        return self.Sigma.shape[0]

    @property
    def samples(self) -> int:
        return self.m * self.n_reps


def _shifts(rng, d, n_reps, qmc_type):
    if qmc_type == "Richtmyer":
        return rng.random((d - 1, n_reps)), None
    return None, rng.integers(0, 2**64, size=(d - 1, n_reps), dtype=np.uint64)


def c1(seed: int = 1) -> Workload:
    """d=10, random correlation (A 10x20), a=-inf, b~U(0,2), Richtmyer 1e4 x 10."""
    rng = np.random.default_rng(seed)
    d = 10
    A = rng.standard_normal((d, 20))
    R = correlation(A @ A.T)
    a = np.full(d, -np.inf)
    b = rng.uniform(0, 2, d)
    sh, _ = _shifts(rng, d, 10, "Richtmyer")
    return Workload("c1_d10_richtmyer", R, a, b, "Richtmyer", 10_000, 10, sh)


def c2(seed: int = 2, d: int = 500, m: int = 2**16, n_reps: int = 12) -> Workload:
    """d=500, random correlation (A 500x600), a~U(-3,-0.5), b~U(0.5,3), Sobol 2^16 x 12."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((d, d + 100))
    R = correlation(A @ A.T)
    a = rng.uniform(-3, -0.5, d)
    b = rng.uniform(0.5, 3, d)
    _, us = _shifts(rng, d, n_reps, "Sobol")
    return Workload(f"c2_d{d}_sobol", R, a, b, "Sobol", m, n_reps, None, us)


def c3(seed: int = 3, d: int = 1000, m: int = 2**17, n_reps: int = 16) -> Workload:
    """d=1000 factor model B B' + diag(psi) (B 1000x20 ~ N(0,0.3^2), psi~U(0.2,1)),
    a=-inf, b=Phi^-1(p), log10 p ~ U(-3,-1); Richtmyer 2^17 x 16."""
    rng = np.random.default_rng(seed)
    B = rng.normal(0, 0.3, (d, 20))
    psi = rng.uniform(0.2, 1.0, d)
    R = correlation(B @ B.T + np.diag(psi))
    a = np.full(d, -np.inf)
    p = 10.0 ** rng.uniform(-3, -1, d)
    b = ndtri(p)
    sh, _ = _shifts(rng, d, n_reps, "Richtmyer")
    return Workload(f"c3_d{d}_factor_richtmyer", R, a, b, "Richtmyer", m, n_reps, sh,
                    extra={"B": B, "psi": psi})


def c3_quarter(seed: int = 3, d: int = 1000, m: int = 2**17, n_reps: int = 16) -> Workload:
    """The c3 covariance with the reference's bound design (+-k sqrt(S_ii),
    P(independent) = 0.25), so that P is O(0.1) and errors are visible."""
    w = c3(seed, d, m, n_reps)
    a, b = bounds_quarter(w.Sigma)
    w.a, w.b = a, b
    w.name = f"c3q_d{d}_factor_quarter_richtmyer"
    return w


def c4(seed: int = 4, n_problems: int = 4096, m: int = 2**14, n_reps: int = 8,
       dmin: int = 16, dmax: int = 256):
    """Batch of problems with d~U{16..256}, A d x (d+8), a~U(-2.5,0), b~U(0,2.5)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_problems):
        d = int(rng.integers(dmin, dmax + 1))
        A = rng.standard_normal((d, d + 8))
        R = correlation(A @ A.T)
        a = rng.uniform(-2.5, 0, d)
        b = rng.uniform(0, 2.5, d)
        _, us = _shifts(rng, d, n_reps, "Sobol")
        out.append(Workload(f"c4_{i}_d{d}", R, a, b, "Sobol", m, n_reps, None, us))
    return out


def c5(seed: int = 5, d: int = 10_000, rho: float = 0.9, m: int = 2**18, n_reps: int = 10,
       bandwidth: int = 64) -> Workload:
    """AR(1) correlation rho^|i-j| at d = 10^4, a=-inf, b~U(-0.5,2.5), Sobol 2^18 x 10;
    the factor is truncated to `bandwidth` super-diagonals."""
    rng = np.random.default_rng(seed)
    idx = np.arange(d)
    R = rho ** np.abs(idx[:, None] - idx[None, :])
    a = np.full(d, -np.inf)
    b = rng.uniform(-0.5, 2.5, d)
    _, us = _shifts(rng, d, n_reps, "Sobol")
    return Workload(f"c5_d{d}_ar1_sobol", R, a, b, "Sobol", m, n_reps, None, us,
                    extra={"bandwidth": bandwidth})

"""Generates the committed fixtures under tests/golden/ (run from the repo root:
``python tests/golden/make_golden.py``).

* ``published.json`` -- values the reference repository publishes for the
  qmc_pnorm! path (its own outputs; the reference cannot run here because
  Julia is absent), each with the file:line it is taken from, plus the
  closed-form value of the same integral (oracle/kat.py).
* ``oracle_cases.npz`` -- small seeded problems (inputs, shifts) with the CPU
  checker's outputs: factor U, perm, permuted bounds, per-shift means, P, 3*SEM.
  GPU tests compare the CUDA path against these fixtures and the live checker.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import kat, oracle as O  # noqa: E402
from dbgenzpaper_b200 import workloads as W  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def sobol_table(dims):
    # the library's own direction numbers, built by a small host routine that
    # does not need a GPU
    import ctypes as C
    from dbgenzpaper_b200 import _lib as L
    V = np.zeros((dims, 32), dtype=np.uint32)
    L.check(L.lib().dbgz_sobol_dirnums(dims, V.ctypes.data_as(C.POINTER(C.c_uint32))))
    return V


def case(name, Sigma, a, b, *, qmc_type, m, n_reps, seed, max_pts=None, cdf_form=0,
         sparse=False, bs=(64, 512)):
    rng = np.random.default_rng(seed)
    d = Sigma.shape[0]
    out = dict(Sigma=Sigma, a_in=a, b_in=b, m=m, n_reps=n_reps,
               max_pts=m if max_pts is None else max_pts, cdf_form=cdf_form, sparse=int(sparse),
               qmc_type=0 if qmc_type == "Richtmyer" else 1, bs1=bs[0], bs2=bs[1])
    if sparse:
        F = O.cholesky_classic(Sigma, a, b, bs[0], bs[1])
    else:
        F = O.cholesky_genz(Sigma, a, b, bs[0], bs[1])
    assert F["rank"] == d
    U = O.truncate_U(F["U"])
    kw = {}
    if qmc_type == "Richtmyer":
        sh = rng.random((d - 1, n_reps))
        out["shifts"] = sh
        kw = dict(shifts=sh)
    else:
        V = sobol_table(d - 1)
        us = rng.integers(0, 2**64, size=(d - 1, n_reps), dtype=np.uint64)
        first = 2 * m
        out.update(V=V, ushifts=us, sobol_first=first)
        kw = dict(qmc_type=O.SOBOL, V=V, ushifts=us, sobol_first=first)
    P, err, npts, reps = O.qmc_pnorm(U, F["a"], F["b"], m=m, n_reps=n_reps,
                                     max_pts=out["max_pts"], max_abs_err=0.0,
                                     cdf_form=cdf_form, sparse=sparse, **kw)
    out.update(U=U, perm=F["perm"], a=F["a"], b=F["b"], scale_vec=F["scale_vec"], reps=reps,
               P=P, err=err, n_pts=npts)
    return {f"{name}/{k}": np.asarray(v) for k, v in out.items()}


def main():
    O.build()
    arrays = {}
    w1 = W.c1()
    arrays.update(case("c1", w1.Sigma, w1.a, w1.b, qmc_type="Richtmyer", m=10_000, n_reps=10,
                       seed=11))
    rng = np.random.default_rng(42)
    S8 = W.rand_spd(8, 4.0, rng)
    arrays.update(case("spd8", S8, np.full(8, -np.inf), np.full(8, 2.0), qmc_type="Richtmyer",
                       m=2**11, n_reps=12, seed=7, max_pts=2**13))
    w2 = W.c2(d=40, m=1024, n_reps=12)
    arrays.update(case("sobol40", w2.Sigma, w2.a, w2.b, qmc_type="Sobol", m=1024, n_reps=12,
                       seed=21))
    T8 = np.diag(np.full(8, 1.8)) + np.diag(np.full(7, 0.25), 1) + np.diag(np.full(7, 0.25), -1)
    arrays.update(case("tridiag8", T8, np.full(8, -np.inf), np.full(8, 1.5), qmc_type="Richtmyer",
                       m=2**11, n_reps=12, seed=21, max_pts=2**13, sparse=True))
    S130 = W.rand_spd(130, 1.0, np.random.default_rng(130))
    lo, up = W.bounds_quarter(S130)
    arrays.update(case("erfc130", S130, lo, up, qmc_type="Richtmyer", m=777, n_reps=6, seed=130,
                       cdf_form=1, bs=(16, 64)))
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **arrays)

    pub = {
        "source": "JakobPeterlin/DBGenzPaper data/sims/table_sparse_dense1.tex (M2 Ultra), "
                  "method DB (qmc_pnorm!, Float64), Sigma_2 = 1 1' + I, bounds +-k sqrt(S_ii), "
                  "k = Phi^-1((1 + 0.25^(1/n))/2)",
        "rows": [],
    }
    # value = median over 20 repetitions, sd = their standard deviation
    for n, m_tot, val, sd, line in ((256, 245760, 0.6981, 3.27e-4, 10),
                                    (512, 245760, 0.7389, 2.84e-4, 20),
                                    (1024, 245760, 0.7738, 2.68e-4, 30),
                                    (2048, 245760, 0.8039, 2.27e-4, 40)):
        S = W.fixed_dense(n)
        lo, up = W.bounds_quarter(S)
        pub["rows"].append(dict(n=n, m_total=m_tot, value=val, sd=sd,
                                cite=f"data/sims/table_sparse_dense1.tex:{line}",
                                closed_form=kat.equicorrelated(1.0, 1.0, lo, up)))
    pub["identity"] = {"value": 0.25, "cite": "results/table_sparse_dense.tex:5-14 (P = 0.2500, SD ~ 1e-16)"}
    with open(os.path.join(HERE, "published.json"), "w") as f:
        json.dump(pub, f, indent=1)


if __name__ == "__main__":
    main()

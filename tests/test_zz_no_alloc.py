"""The allocation-free pass, dbgz_pnorm_pass_noalloc, against dbgz_pnorm.

Some callers cannot let a library allocate device memory: frameworks that
own every device buffer and hand them to the library (an XLA/JAX custom
call, a Julia program whose GPU memory is CUDA.jl's pool), and
latency-critical callers for whom cudaMalloc/cudaFree would synchronise the
whole device.  They call dbgz_pnorm_pass_noalloc with device pointers they
own; its scratch is a fixed array inside the library.

This test calls it through the C ABI twice in a row, on two different
problems (the second larger, so it runs on the array's leftovers from the
first), and checks each result against the allocating entry point at the
FP64 tolerance the other tests use.  The file name makes pytest collect it
last, so a run that stops at the first failure has run every other test
before it.
"""
import numpy as np
import pytest

from dbgenzpaper_b200 import workloads as W
from dbgenzpaper_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _pass_both_ways(D, torch, n, m, n_reps, seed):
    rng = np.random.default_rng(seed)
    S = W.rand_spd(n, 1.0, rng)
    lo, up = W.bounds_quarter(S)
    sh = rng.random((n - 1, n_reps))
    Q = D.QMCData(S, lo, up, D.QMC_opts(m=m, n_reps=n_reps, max_pts=m, max_abs_err=0.0),
                  shifts=sh)
    _, _, _, reps_ref = D.qmc_pnorm(Q, precision=L.PREC_FP64, return_reps=True)
    F = Q.C
    dev = torch.device("cuda", 0)

    def dev_f64(x):  # column-major flattening, copied into caller-owned memory
        return torch.from_numpy(np.ascontiguousarray(np.ravel(x, order="F"), dtype=np.float64)).to(dev)

    U, a, b = dev_f64(F.U), dev_f64(F.a), dev_f64(F.b)
    q, shifts = dev_f64(D.get_sqrt_primes(n - 1)), dev_f64(sh)
    out = torch.full((n_reps,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = L.lib().dbgz_pnorm_pass_noalloc(n, U.data_ptr(), a.data_ptr(), b.data_ptr(), q.data_ptr(),
                                         shifts.data_ptr(), m, n_reps, 0, out.data_ptr(), stream)
    assert st == L.OK
    torch.cuda.synchronize(dev)
    np.testing.assert_allclose(out.cpu().numpy(), reps_ref, rtol=1e-12, atol=0)


def test_noalloc_pass_matches_pnorm_twice(dbgz):
    import torch
    dbgz.get_context(0)
    _pass_both_ways(dbgz, torch, n=37, m=1000, n_reps=6, seed=37)
    _pass_both_ways(dbgz, torch, n=300, m=2500, n_reps=4, seed=300)


def test_noalloc_rejects_sizes_beyond_its_array(dbgz):
    lib = L.lib()
    fake = 256  # never dereferenced: the size checks come first
    assert lib.dbgz_pnorm_pass_noalloc(8193, fake, fake, fake, fake, fake, 100, 2, 0, fake,
                                       None) == L.ERR_DIMENSION
    assert lib.dbgz_pnorm_pass_noalloc(10, fake, fake, fake, fake, fake, 128 * 131072, 2, 0, fake,
                                       None) == L.ERR_DIMENSION
    assert lib.dbgz_pnorm_pass_noalloc(10, None, fake, fake, fake, fake, 100, 2, 0, fake,
                                       None) == L.ERR_INVALID_ARGUMENT
    # tile counts whose product (or m + 127) would wrap in 64 bits
    assert lib.dbgz_pnorm_pass_noalloc(10, fake, fake, fake, fake, fake, 384, 6148914691236517206, 0,
                                       fake, None) == L.ERR_DIMENSION
    assert lib.dbgz_pnorm_pass_noalloc(10, fake, fake, fake, fake, fake, 2**63 - 1, 1, 0, fake,
                                       None) == L.ERR_DIMENSION

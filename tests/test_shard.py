"""Multi-GPU sharding logic on CPU: two gloo ranks own disjoint shift blocks
and one all-gather rebuilds the per-shift means in order (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dbgenzpaper_b200 import shard


def test_shift_blocks_partition():
    for n in (1, 7, 16, 33):
        for w in (1, 2, 3, 8):
            blocks = [shard.shift_block(r, w, n) for r in range(w)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(a1 == b0 for (_, a1), (b0, _) in zip(blocks, blocks[1:]))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shift_block(2, 2, 4)


def test_combine_matches_reference_formula():
    reps = np.array([0.25, 0.2501, 0.2499, 0.25002])
    P, e = shard.combine(reps)
    n = reps.size
    sd = np.sqrt(np.sum((reps - reps.mean()) ** 2 / n) / (n - 1))
    assert abs(P - reps.mean()) < 1e-16 and abs(e - 3 * sd) < 1e-16


def _worker(rank, world, port, n_total, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    a, b = shard.shift_block(rank, world, n_total)
    local = np.arange(a, b, dtype=np.float64) * 0.01 + 0.2
    allr = shard.gather_reps(local, n_total)
    q.put((rank, allr.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("n_total", [16, 9])
def test_gather_two_ranks_gloo(n_total):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_total, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = (np.arange(n_total) * 0.01 + 0.2).tolist()
    assert out[0] == want and out[1] == want


def _estimator_worker(rank, world, port, case, q):
    """One rank: the checker's qmc_pnorm! over this rank's shift block of the
    problem, then the all-gather of the per-shift means."""
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    U, a, b, kw, n_total = case
    s0, s1 = shard.shift_block(rank, world, n_total)
    kw = dict(kw)
    if "shifts" in kw:
        kw["shifts"] = kw["shifts"][:, s0:s1]
    else:
        kw["ushifts"] = kw["ushifts"][:, s0:s1]
    local = O.qmc_pnorm(U, a, b, n_reps=s1 - s0, **kw)[3]
    allr = shard.gather_reps(local, n_total)
    q.put((rank, allr.tobytes()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("gen,world", [("Richtmyer", 2), ("Sobol", 2), ("Richtmyer", 3)])
def test_sharded_estimator_equals_single_process(oracle, gen, world):
    """Ranks that each integrate their own block of shifts (no data-path
    communication) and all-gather the per-shift means reproduce the
    single-process qmc_pnorm! per-shift means and P bit for bit
    (src/qmc.jl:328: the shifts are independent; :814-815: mean and 3 SEM)."""
    from dbgenzpaper_b200 import workloads as W
    rng = np.random.default_rng(7)
    n, m, R = 24, 700, 11
    S = W.rand_spd(n, 1.0, rng)
    lo, up = W.bounds_quarter(S)
    F = oracle.cholesky_genz(S, lo, up)
    U = oracle.truncate_U(F["U"])
    kw = dict(m=m, max_pts=3 * m, max_abs_err=0.0)  # three passes, no tolerance stop
    if gen == "Richtmyer":
        kw["shifts"] = np.asfortranarray(rng.random((n - 1, R)))
    else:
        import dbgenzpaper_b200 as D
        kw.update(qmc_type=oracle.SOBOL, V=D.sobol_dirnums(n - 1), sobol_first=D.sobol_first_index(m),
                  ushifts=np.asfortranarray(rng.integers(0, 2**64, size=(n - 1, R), dtype=np.uint64)))
    P1, e1, n1, reps1 = oracle.qmc_pnorm(U, F["a"], F["b"], n_reps=R, **kw)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    case = (U, F["a"], F["b"], kw, R)
    procs = [ctx.Process(target=_estimator_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        reps = np.frombuffer(out[r], dtype=np.float64)
        assert np.array_equal(reps, reps1)
        P, e = shard.combine(reps)
        assert P == P1 and e == e1

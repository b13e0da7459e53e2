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

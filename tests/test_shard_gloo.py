"""The multi-GPU layout of the batch: N ranks each build a contiguous shard of one list
of N * 512 independent matrices (clspmv_b200.matrices.shard / batch_mixed(first, n)),
with no collective on the data path.  Checked here with two gloo ranks on the CPU: the
shards are disjoint, cover the list, and every matrix is the one a single process
builds at that position."""
import os
import socket

import numpy as np
import pytest

from clspmv_b200 import matrices as M


def _digest(gen):
    return [(k, h, w, int(r.size), int(np.sum(r.astype(np.int64) * 31 + c)), float(np.sum(v, dtype=np.float64)))
            for k, h, w, r, c, v in gen]


def _rank(rank, world, port, total, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, n = M.shard(total, world, rank)
        mine = _digest(M.batch_mixed(total, lo=50, hi=400, seed=7, first=first, n=n))
        got = [None] * world
        dist.all_gather_object(got, (first, n, mine))
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("total", [10, 11])
def test_two_rank_shards_rebuild_the_list(total):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, total, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = _digest(M.batch_mixed(total, lo=50, hi=400, seed=7))
    (f0, n0, s0), (f1, n1, s1) = got
    assert (f0, f1) == (0, n0) and n0 + n1 == total and abs(n0 - n1) <= 1
    assert s0 + s1 == whole


def test_shard_arithmetic():
    for total in (0, 1, 7, 512, 1024, 1000):
        for world in (1, 2, 3, 8):
            parts = [M.shard(total, world, r) for r in range(world)]
            assert sum(n for _, n in parts) == total
            assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    with pytest.raises(ValueError):
        M.shard(10, 2, 2)

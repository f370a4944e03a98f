"""Host side of the multi-GPU path, on CPU with two gloo ranks: cost-balanced
sharding of a job list and the max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest

from benchntt_b200 import dist as D
from benchntt_b200 import workloads as W


def test_shard_covers_every_job_once_and_balances():
    b = W.uneven_batch()
    for world in (1, 2, 3, 8):
        parts = D.shard_by_cost(b.logns, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(b.count))
        loads = [int(D.transform_cost(b.logns[p]).sum()) for p in parts]
        # the 2^20 transforms are the largest indivisible units
        assert max(loads) - min(loads) <= int(D.transform_cost([20])[0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    d = D.Dist(backend="gloo", timeout_s=60)
    try:
        b = W.uneven_batch(n_small=5000, large=((16, 3), (20, 1)))
        mine = D.shard_by_cost(b.logns, d.world)[d.rank]
        # each rank's own time; the job-wide time is the slowest rank's
        t = 1.0 + rank
        tmax = d.max(t)
        total = d.sum(float(len(mine)))
        d.barrier()
        q.put((rank, tmax, total, len(mine)))
    finally:
        d.close()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.0, 2.0]          # max over ranks on both
    assert res[0][2] == res[1][2] == 5004.0           # every job counted once
    assert res[0][3] + res[1][3] == 5004

"""Host side of the multi-GPU path, on CPU with two gloo ranks: cost-balanced
sharding of a job list, the max-over-ranks timing reduction, and a split
job list computed rank by rank (each rank runs its shard through the oracle,
as a GPU rank runs it through its own batch) whose union equals the one-rank
result bit for bit."""
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


def test_library_split_matches_python_shard():
    """bntt_split_by_cost (the C ABI, no GPU needed) and dist.shard_by_cost
    give every job the same owner."""
    import benchntt_b200 as bn
    b = W.uneven_batch()
    for world in (1, 2, 3, 4, 8):
        owner = bn.split_by_cost(b.logns, world)
        for r, part in enumerate(D.shard_by_cost(b.logns, world)):
            assert (owner[part] == r).all()
        assert owner.max() < world


SPLIT_BATCH = dict(seed=11, n_small=600, large=((12, 3), (14, 2), (16, 1)))


def _split_inputs(b):
    import common as C
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in b.sizes}
    xs = [C.uniform_pairs(W.SEED_INPUT + i, 1 << int(n), C.Q_NTT) for i, n in enumerate(b.logns)]
    return tables, xs


def _split_worker(rank, world, port, q):
    import common as C
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    d = D.Dist(backend="gloo", timeout_s=60)
    try:
        b = W.uneven_batch(**SPLIT_BATCH)
        tables, xs = _split_inputs(b)
        mine = D.shard_by_cost(b.logns, d.world)[d.rank]
        ys = C.oracle_ntt_jobs([xs[i] for i in mine], [tables[int(b.logns[i])] for i in mine],
                               [int(b.logns[i]) for i in mine])
        work = float(D.transform_cost(b.logns[mine]).sum())
        total = d.sum(work)
        d.barrier()
        q.put((rank, [int(i) for i in mine], ys, work, total))
    finally:
        d.close()


def test_split_job_list_computed_on_two_ranks_equals_one_rank():
    import common as C
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(2)), key=lambda r: r[0])
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    b = W.uneven_batch(**SPLIT_BATCH)
    tables, xs = _split_inputs(b)
    whole = C.oracle_ntt_jobs(xs, [tables[int(n)] for n in b.logns], [int(n) for n in b.logns])
    seen = np.zeros(b.count, dtype=int)
    for rank, mine, ys, work, total in res:
        assert total == float(D.transform_cost(b.logns).sum())
        for i, y in zip(mine, ys):
            seen[i] += 1
            assert np.array_equal(y, whole[i]), f"job {i} (2^{b.logns[i]}) on rank {rank}"
    assert (seen == 1).all(), "every job computed by exactly one rank"
    # the split is balanced to within the largest job
    works = [r[3] for r in res]
    assert max(works) - min(works) <= int(D.transform_cost([16])[0])

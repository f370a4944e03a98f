"""One job list over several batches (bntt_multi_*), each batch on its own
context with its own copy of the plans' tables.  On a one-GPU box the two
contexts share device 0; their kernels are independent (no kernel waits on
another's), which is what several devices run.  Bit-exact against the oracle
and against one batch running the whole list."""
import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W

pytestmark = pytest.mark.gpu

SIZES = list(range(1, 11)) + [12, 16, 20]


def make(ctx):
    plans = [bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT))
             for n in SIZES]
    return plans, bn.Batch(ctx, plans)


def host_jobs(logns, x, y):
    offs = np.concatenate([[0], np.cumsum([1 << int(n) for n in logns])[:-1]]).astype(np.int64) * 16
    pid = {n: i for i, n in enumerate(SIZES)}
    return bn.Batch.jobs([x.ctypes.data + int(o) for o in offs], [y.ctypes.data + int(o) for o in offs],
                         [pid[int(n)] for n in logns]), offs // 16


@pytest.mark.parametrize("parts", [1, 2, 3])
def test_multi_run_host_equals_one_batch_and_oracle(parts):
    b = W.uneven_batch(seed=31, n_small=4000, small_lo=1, large=((12, 5), (16, 2), (20, 1)))
    x = C.uniform_pairs(W.SEED_INPUT, b.total, C.Q_NTT)
    ctxs = [bn.Context(0) for _ in range(parts)]
    made = [make(c) for c in ctxs]
    multi = bn.Multi([m[1] for m in made])
    y = np.zeros_like(x)
    jobs, offs = host_jobs(b.logns, x, y)
    owner = multi.split(jobs)
    assert np.array_equal(owner, bn.split_by_cost(b.logns, parts))
    assert set(np.unique(owner)) == set(range(parts))
    multi.run_host(jobs)
    # one batch over the whole list
    y1 = np.zeros_like(x)
    jobs1, _ = host_jobs(b.logns, x, y1)
    made[0][1].run_host(jobs1)
    assert np.array_equal(y, y1)
    # the oracle, job by job, on a sample that covers every size
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in SIZES}
    pick = [i for i in range(b.count) if b.logns[i] >= 12 or i % 97 == 0]
    want = C.oracle_ntt_jobs([x[offs[i]:offs[i] + (1 << int(b.logns[i]))] for i in pick],
                             [tables[int(b.logns[i])] for i in pick], [int(b.logns[i]) for i in pick],
                             threads=8)
    for i, w in zip(pick, want):
        assert np.array_equal(y[offs[i]:offs[i] + (1 << int(b.logns[i]))], w), f"job {i}"
    multi.close()
    for plans, batch in made:
        batch.close()
        for p in plans:
            p.close()
    for c in ctxs:
        c.close()


def test_multi_rejects_mismatched_batches():
    c1, c2 = bn.Context(0), bn.Context(0)
    p1, b1 = make(c1)
    q = bn.Plan(c2, 5, C.Q_NTT, C.MU_NTT, C.uniform_pairs(1, 32, C.Q_NTT))
    b2 = bn.Batch(c2, [q])
    L = bn.lib()
    import ctypes
    h = ctypes.c_void_p()
    arr = (ctypes.c_void_p * 2)(b1.handle.value, b2.handle.value)
    assert L.bntt_multi_create(ctypes.byref(h), arr, 2) == bn.EINVAL
    arr = (ctypes.c_void_p * 2)(b1.handle.value, b1.handle.value)
    assert L.bntt_multi_create(ctypes.byref(h), arr, 2) == bn.EINVAL
    b1.close()
    b2.close()
    for p in p1 + [q]:
        p.close()
    c1.close()
    c2.close()

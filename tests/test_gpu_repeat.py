"""Repeated runs give identical bytes (a check for exchange races).

The tile kernels synchronise only within a warp between passes whose data
stay inside each warp, and the persistent kernels hand tiles between CTAs
through counters; a missing barrier would show as runs that differ from one
another.  Each case runs the same call several times, compares every
output with the first bit for bit, and the first with the oracle.
"""
import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
REPEATS = 6


@pytest.fixture(scope="module")
def ctx():
    c = bn.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("logn,batch", [(6, 4096), (8, 4096), (9, 2048), (10, 2048), (16, 16)])
@pytest.mark.parametrize("direction", ["forward", "inverse"])
def test_plan_runs_repeat_bit_exact(ctx, logn, batch, direction):
    n = 1 << logn
    t = C.uniform_pairs(5000 + logn, n, C.Q_NTT)
    x = C.uniform_pairs(6000 + logn, batch * n, C.Q_NTT)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    fn = bn.lib().bntt_ntt_forward_dev if direction == "forward" else bn.lib().bntt_ntt_inverse_dev
    dx, dy = DevBuf.from_array(ctx, x), DevBuf(ctx, x.nbytes)
    first = None
    for _ in range(REPEATS):
        bn.check(fn(p.handle, dy.ptr, dx.ptr, batch))
        out = dy.to_array(batch * n)
        if first is None:
            first = out
            want = (C.oracle_ntt(x[:n], t, logn) if direction == "forward"
                    else C.oracle_ntt_inverse(x[:n], t, logn))
            assert np.array_equal(first[:n], want)
        else:
            assert np.array_equal(out, first)
    dx.free()
    dy.free()
    p.close()


@pytest.mark.parametrize("direction", ["forward", "inverse"])
def test_batch_runs_repeat_bit_exact(ctx, direction):
    b = W.uneven_batch(seed=34, n_small=20000, large=((16, 4), (20, 1)))
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in b.sizes}
    plans = {n: bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, tables[n]) for n in b.sizes}
    pid = {n: i for i, n in enumerate(b.sizes)}
    eng = bn.Batch(ctx, [plans[n] for n in b.sizes])
    x = C.uniform_pairs(W.SEED_INPUT + 1, b.total, C.Q_NTT)
    dx, dy = DevBuf.from_array(ctx, x), DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs([dx.addr + o for o in offs], [dy.addr + o for o in offs],
                         [pid[int(n)] for n in b.logns])
    run = eng.run_dev if direction == "forward" else eng.run_inverse_dev
    first = None
    for _ in range(REPEATS):
        run(jobs)
        assert eng.status() == bn.OK
        out = dy.to_array(b.total)
        if first is None:
            first = out
        else:
            assert np.array_equal(out, first)
    # one job of each size against the oracle
    for n in b.sizes:
        i = int(np.nonzero(b.logns == n)[0][0])
        o = int(b.offsets[i])
        xi = x[o:o + (1 << n)]
        want = (C.oracle_ntt(xi, tables[n], n) if direction == "forward"
                else C.oracle_ntt_inverse(xi, tables[n], n))
        assert np.array_equal(first[o:o + (1 << n)], want), f"2^{n}"
    eng.close()
    for p in plans.values():
        p.close()
    dx.free()
    dy.free()

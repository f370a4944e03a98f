"""The batch run that allocates no device memory (bntt_batch_run_dev_noalloc).

It is for callers that cannot call cudaMalloc when they submit work, e.g.
because another allocator's pool already owns the GPU's memory or because an
allocation would stall a latency-critical path.  Its scratch lives in a fixed
4 MiB array inside the library.  These checks call it through the C ABI and
compare it with bntt_batch_run_dev, bit for bit (integer results: tolerance
0), on two calls in a row -- the second call must not see leftovers of the
first -- and confirm the context's device allocations do not change.

This file is collected last so a failure here does not hide other results;
it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_twice():
    ctx = bn.Context(0)
    batch = W.uneven_batch(seed=21, n_small=3000, large=((12, 2), (16, 1)))
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in batch.sizes}
    plans = {n: bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, tables[n]) for n in batch.sizes}
    pid = {n: i for i, n in enumerate(batch.sizes)}
    engine = bn.Batch(ctx, [plans[n] for n in batch.sizes])
    x = C.uniform_pairs(W.SEED_INPUT, batch.total, C.Q_NTT)
    dx = DevBuf.from_array(ctx, x)
    dy_ref = DevBuf(ctx, batch.total * 16)
    dy = DevBuf(ctx, batch.total * 16)
    offs = [16 * int(o) for o in batch.offsets]
    ids = [pid[int(n)] for n in batch.logns]
    jobs_ref = bn.Batch.jobs([dx.addr + o for o in offs], [dy_ref.addr + o for o in offs], ids)
    jobs = bn.Batch.jobs([dx.addr + o for o in offs], [dy.addr + o for o in offs], ids)

    engine.run_dev(jobs_ref)
    assert engine.status() == bn.OK
    want = dy_ref.to_array()

    L = bn.lib()
    in_use = ctx.hbm_in_use
    for call in range(2):
        zero = np.zeros((batch.total, 2), dtype=np.uint64)  # fresh output each call
        bn.check(L.bntt_copy_h2d(ctx.handle, dy.ptr, zero.ctypes.data, zero.nbytes))
        bn.check(L.bntt_batch_run_dev_noalloc(engine.handle, jobs, len(jobs)))
        got = dy.to_array()
        assert np.array_equal(got, want), f"call {call + 1} differs from bntt_batch_run_dev"
        assert ctx.hbm_in_use == in_use, "the no-allocation path allocated device memory"

    # a schedule larger than the fixed scratch is refused before any work
    many = 120_000
    big = bn.Batch.jobs([dx.addr] * many, [dy.addr] * many, [pid[4]] * many)
    rc = L.bntt_batch_run_dev_noalloc(engine.handle, big, many)
    assert rc == bn.EINVAL
    assert b"scratch" in L.bntt_last_error()

    for d in (dx, dy, dy_ref):
        d.free()
    engine.close()
    for p in plans.values():
        p.close()
    ctx.close()

"""The batch run that allocates no device memory (bntt_batch_run_dev_noalloc).

It is for callers that cannot call cudaMalloc when they submit work, e.g.
because another allocator's pool already owns the GPU's memory or because an
allocation would stall a latency-critical path.  Its scratch lives in a fixed
4 MiB array inside the library.  These checks call it through the C ABI and
compare it with bntt_batch_run_dev, bit for bit (integer results: tolerance
0), on calls in a row -- a later call must not see leftovers of an earlier
one, also when the later list is smaller and has different large jobs -- and
confirm that neither the context's allocations nor the device's free memory
(cudaMemGetInfo) change across the calls.

This file is collected last so a failure here does not hide other results;
it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu


def _free_bytes() -> int:
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


class _Lists:
    """Two job lists over one set of plans: the uneven mix of 3,000 small
    transforms with 2 x 2^12 and 1 x 2^16, and a smaller list of three 2^16
    transforms followed by one 2^20."""

    def __init__(self, ctx):
        self.ctx = ctx
        sizes = list(range(4, 11)) + [12, 16, 20]
        self.pid = {n: i for i, n in enumerate(sizes)}
        self.plans = [bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT,
                              C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT)) for n in sizes]
        self.engine = bn.Batch(ctx, self.plans)
        mix = W.uneven_batch(seed=21, n_small=3000, large=((12, 2), (16, 1)))
        self.lists = [[int(n) for n in mix.logns], [16, 16, 16, 20]]
        total = max(sum(1 << n for n in l) for l in self.lists)
        self.dx = DevBuf.from_array(ctx, C.uniform_pairs(W.SEED_INPUT, total, C.Q_NTT))
        self.dy_ref = DevBuf(ctx, total * 16)
        self.dy = DevBuf(ctx, total * 16)

    def jobs(self, k: int, out: DevBuf):
        logns = self.lists[k]
        offs = np.concatenate([[0], np.cumsum([1 << n for n in logns])[:-1]]) * 16
        return bn.Batch.jobs([self.dx.addr + int(o) for o in offs], [out.addr + int(o) for o in offs],
                             [self.pid[n] for n in logns]), sum(1 << n for n in logns)

    def close(self):
        for d in (self.dx, self.dy, self.dy_ref):
            d.free()
        self.engine.close()
        for p in self.plans:
            p.close()


def test_noalloc_matches_allocating_entry_point_on_calls_in_a_row():
    ctx = bn.Context(0)
    t = _Lists(ctx)
    L = bn.lib()
    want = []
    for k in range(2):
        jobs, rows = t.jobs(k, t.dy_ref)
        t.engine.run_dev(jobs)
        assert t.engine.status() == bn.OK
        want.append(t.dy_ref.to_array(rows))

    in_use = ctx.hbm_in_use
    free0 = None
    # the first list twice, then the smaller list with other large jobs
    for call, k in enumerate((0, 0, 1)):
        jobs, rows = t.jobs(k, t.dy)
        zero = np.zeros((rows, 2), dtype=np.uint64)  # fresh output each call
        bn.check(L.bntt_copy_h2d(ctx.handle, t.dy.ptr, zero.ctypes.data, zero.nbytes))
        bn.check(L.bntt_batch_run_dev_noalloc(t.engine.handle, jobs, len(jobs)))
        assert t.engine.last_launches == 1
        assert t.engine.status() == bn.OK, "status after a no-allocation run"
        got = t.dy.to_array(rows)
        assert np.array_equal(got, want[k]), f"call {call + 1} differs from bntt_batch_run_dev"
        assert ctx.hbm_in_use == in_use, "the no-allocation path allocated through the context"
        if free0 is None:
            # the first call may load the library's module that holds the
            # array; every later call must leave the device's free memory alone
            free0 = _free_bytes()
        else:
            assert _free_bytes() == free0, "device free memory changed across a no-allocation call"

    # an empty list launches nothing and reports no launch
    bn.check(L.bntt_batch_run_dev_noalloc(t.engine.handle, bn.Batch.jobs([], [], []), 0))
    assert t.engine.last_launches == 0

    # a schedule larger than the fixed scratch is refused before any work
    many = 120_000
    big = bn.Batch.jobs([t.dx.addr] * many, [t.dy.addr] * many, [t.pid[4]] * many)
    rc = L.bntt_batch_run_dev_noalloc(t.engine.handle, big, many)
    assert rc == bn.EINVAL
    assert b"scratch" in L.bntt_last_error()
    t.close()
    ctx.close()


def test_noalloc_refused_while_the_stream_is_captured():
    from cuda.bindings import runtime as rt
    ctx = bn.Context(0)
    t = _Lists(ctx)
    jobs, rows = t.jobs(1, t.dy)
    L = bn.lib()
    stream = rt.cudaStream_t(ctx.stream)
    err, = rt.cudaStreamBeginCapture(stream, rt.cudaStreamCaptureMode.cudaStreamCaptureModeThreadLocal)
    assert err == rt.cudaError_t.cudaSuccess
    rc = L.bntt_batch_run_dev_noalloc(t.engine.handle, jobs, len(jobs))
    err, graph = rt.cudaStreamEndCapture(stream)
    assert err == rt.cudaError_t.cudaSuccess, "the refused call invalidated the capture"
    rt.cudaGraphDestroy(graph)
    assert rc == bn.EINVAL
    assert b"captured" in L.bntt_last_error()
    # the stream is usable afterwards and the call then runs normally
    t.engine.run_dev(jobs)
    want = t.dy.to_array(rows)
    zero = np.zeros((rows, 2), dtype=np.uint64)
    bn.check(L.bntt_copy_h2d(ctx.handle, t.dy.ptr, zero.ctypes.data, zero.nbytes))
    bn.check(L.bntt_batch_run_dev_noalloc(t.engine.handle, jobs, len(jobs)))
    assert np.array_equal(t.dy.to_array(rows), want)
    t.close()
    ctx.close()

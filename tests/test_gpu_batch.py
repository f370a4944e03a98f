"""GPU parity of the persistent mixed-size batch engine (bntt_batch_*).

Every job of a batch must equal the reference transform of its input
(bit-exact); the same job must give the same bytes alone and inside a mix;
graph replays and schedule rebuilds must not change results.
"""
import ctypes
import hashlib

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")


@pytest.fixture(scope="module")
def ctx():
    c = bn.Context(0)
    yield c
    c.close()


class Setup:
    """Plans for every size of a workload, packed device input/output."""

    def __init__(self, ctx, batch: W.Batch, q=C.Q_NTT, mu=C.MU_NTT, seed=W.SEED_INPUT):
        self.ctx, self.batch = ctx, batch
        self.tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, q) for n in batch.sizes}
        self.plans = {n: bn.Plan(ctx, n, q, mu, self.tables[n]) for n in batch.sizes}
        self.plan_ids = {n: i for i, n in enumerate(batch.sizes)}
        self.x = C.uniform_pairs(seed, batch.total, q)
        self.dx = DevBuf.from_array(ctx, self.x)
        self.dy = DevBuf(ctx, batch.total * 16)
        self.engine = bn.Batch(ctx, [self.plans[n] for n in batch.sizes])

    def jobs(self, idx=None, inplace=False):
        idx = range(self.batch.count) if idx is None else idx
        xs = [self.dx.addr + 16 * int(self.batch.offsets[i]) for i in idx]
        ys = xs if inplace else [self.dy.addr + 16 * int(self.batch.offsets[i]) for i in idx]
        return bn.Batch.jobs(xs, ys, [self.plan_ids[int(self.batch.logns[i])] for i in idx])

    def output(self):
        return self.dy.to_array(self.batch.total)

    def expected(self, threads=8):
        b = self.batch
        xs = [self.x[o:o + (1 << n)] for o, n in zip(b.offsets, b.logns)]
        ts = [self.tables[int(n)] for n in b.logns]
        return np.concatenate(C.oracle_ntt_jobs(xs, ts, [int(n) for n in b.logns], threads=threads))

    def close(self):
        self.engine.close()
        for p in self.plans.values():
            p.close()
        self.dx.free()
        self.dy.free()


def test_mixed_small_sizes(ctx):
    b = W.uneven_batch(seed=1, n_small=3000, small_lo=1, small_hi=10, large=())
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    assert s.engine.status() == bn.OK
    # a new job list: the device-side schedule build, then the persistent kernel
    assert s.engine.last_launches == 2
    assert np.array_equal(s.output(), s.expected())
    # the same list again: one graph replay of the persistent kernel
    zero = np.zeros((b.total, 2), dtype=np.uint64)
    bn.check(bn.lib().bntt_copy_h2d(ctx.handle, s.dy.ptr, zero.ctypes.data, zero.nbytes))
    s.engine.run_dev(s.jobs())
    assert s.engine.status() == bn.OK
    assert s.engine.last_launches == 1
    assert np.array_equal(s.output(), s.expected())
    s.close()


def test_mixed_with_large_transforms(ctx):
    b = W.uneven_batch(seed=2, n_small=2000, large=((11, 3), (13, 2), (16, 3), (20, 1)))
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    assert s.engine.status() == bn.OK
    assert np.array_equal(s.output(), s.expected())
    s.close()


@pytest.mark.parametrize("logn", [16, 20])
def test_large_job_matches_reference_fixture(ctx, logn):
    """A 2^16 / 2^20 job inside a mix equals the compiled reference's output
    on the fixture inputs (SHA-256 in tests/golden/ref_gen.npz)."""
    n = 1 << logn
    x = C.uniform_pairs(1000 + logn, n, C.Q_NTT)
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    small_t = C.uniform_pairs(5, 1024, C.Q_NTT)
    p_big = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    p_small = bn.Plan(ctx, 10, C.Q_NTT, C.MU_NTT, small_t)
    eng = bn.Batch(ctx, [p_big, p_small])
    dx = DevBuf.from_array(ctx, x)
    dy = DevBuf(ctx, n * 16)
    xs_small = C.uniform_pairs(6, 1024 * 300, C.Q_NTT)
    dxs = DevBuf.from_array(ctx, xs_small)
    dys = DevBuf(ctx, xs_small.nbytes)
    jobs = bn.Batch.jobs([dx.addr] + [dxs.addr + 16384 * i for i in range(300)],
                         [dy.addr] + [dys.addr + 16384 * i for i in range(300)], [0] + [1] * 300)
    eng.run_dev(jobs)
    assert eng.status() == bn.OK
    y = dy.to_array()
    assert hashlib.sha256(y.astype("<u8").tobytes()).hexdigest() == str(GEN[f"ntt_sha_{logn}"])
    assert np.array_equal(dys.to_array(), C.oracle_ntt(xs_small, small_t, 10, threads=8, form=1))
    for d in (dx, dy, dxs, dys):
        d.free()
    eng.close()
    p_big.close()
    p_small.close()


def test_job_alone_equals_job_in_mix(ctx):
    b = W.uneven_batch(seed=3, n_small=1500, large=((16, 2), (20, 1)))
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    mixed = s.output()
    for i in [0, 7, int(np.argmax(b.logns)), b.count - 1]:
        s.engine.run_dev(s.jobs([i]))
        assert s.engine.status() == bn.OK
        o, n = int(b.offsets[i]), 1 << int(b.logns[i])
        assert np.array_equal(s.output()[o:o + n], mixed[o:o + n])
    s.close()


def test_graph_replay_and_rebuild(ctx):
    b = W.uneven_batch(seed=4, n_small=800, large=((12, 2),))
    s = Setup(ctx, b)
    want = s.expected()
    jobs = s.jobs()
    for _ in range(3):           # replay of the cached schedule
        s.dy.ctx.synchronize()
        s.engine.run_dev(jobs)
        assert np.array_equal(s.output(), want)
    sub = s.jobs(list(range(0, b.count, 3)))  # a different list rebuilds
    s.engine.run_dev(sub)
    assert s.engine.status() == bn.OK
    s.engine.run_dev(jobs)
    assert np.array_equal(s.output(), want)
    s.close()


def test_in_place_jobs(ctx):
    b = W.uneven_batch(seed=5, n_small=500, large=((14, 1),))
    s = Setup(ctx, b)
    want = s.expected()
    s.engine.run_dev(s.jobs(inplace=True))
    assert s.engine.status() == bn.OK
    assert np.array_equal(s.dx.to_array(b.total), want)
    s.close()


def test_run_host(ctx):
    b = W.uneven_batch(seed=6, n_small=600, large=((16, 1),))
    s = Setup(ctx, b)
    y = np.zeros_like(s.x)
    xs = [s.x.ctypes.data + 16 * int(o) for o in b.offsets]
    ys = [y.ctypes.data + 16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs(xs, ys, [s.plan_ids[int(n)] for n in b.logns])
    s.engine.run_host(jobs)
    assert np.array_equal(y, s.expected())
    s.close()


def test_u128_layout_batch_forward_and_inverse(ctx):
    """Plans in the little-endian u128 layout (the persistent kernels are
    compiled once per layout): a mix of 2^1..2^10 plus 2^12 and 2^16 jobs,
    forward and inverse, equal the oracle on the same values."""
    b = W.uneven_batch(seed=33, n_small=1500, small_lo=1, small_hi=10, large=((12, 2), (16, 1)))
    tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in b.sizes}
    plans = {n: bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, tables[n][:, ::-1].copy(), bn.LAYOUT_U128)
             for n in b.sizes}
    pid = {n: i for i, n in enumerate(b.sizes)}
    eng = bn.Batch(ctx, [plans[n] for n in b.sizes])
    x = C.uniform_pairs(W.SEED_INPUT, b.total, C.Q_NTT)
    dx = DevBuf.from_array(ctx, x[:, ::-1].copy())
    dy = DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs([dx.addr + o for o in offs], [dy.addr + o for o in offs],
                         [pid[int(n)] for n in b.logns])
    xs = [x[int(o):int(o) + (1 << int(n))] for o, n in zip(b.offsets, b.logns)]
    ts = [tables[int(n)] for n in b.logns]
    eng.run_dev(jobs)
    assert eng.status() == bn.OK
    want = np.concatenate(C.oracle_ntt_jobs(xs, ts, [int(n) for n in b.logns], threads=8))
    assert np.array_equal(dy.to_array(b.total)[:, ::-1], want)
    eng.run_inverse_dev(jobs)
    assert eng.status() == bn.OK
    got = dy.to_array(b.total)[:, ::-1]
    for i in range(b.count):
        o, n = int(b.offsets[i]), int(b.logns[i])
        assert np.array_equal(got[o:o + (1 << n)], C.oracle_ntt_inverse(x[o:o + (1 << n)], tables[n], n)), \
            f"job {i} (2^{n})"
    eng.close()
    for p in plans.values():
        p.close()
    dx.free()
    dy.free()


def test_reference_arith_batch():
    c = bn.Context(0, arith=bn.ARITH_REFERENCE)
    b = W.uneven_batch(seed=7, n_small=400, large=((12, 1),))
    s = Setup(c, b)
    s.engine.run_dev(s.jobs())
    assert np.array_equal(s.output(), s.expected())
    s.close()
    c.close()


def test_invalid_jobs(ctx):
    b = W.uneven_batch(seed=8, n_small=10, large=())
    s = Setup(ctx, b)
    jobs = s.jobs()
    jobs[3].plan = 99
    with pytest.raises(bn.BnttError) as e:
        s.engine.run_dev(jobs)
    assert e.value.status == bn.EINVAL
    jobs = s.jobs()
    jobs[2].x = s.dx.addr + 8
    with pytest.raises(bn.BnttError):
        s.engine.run_dev(jobs)
    s.engine.run_dev(s.jobs())  # valid again
    assert s.engine.status() == bn.OK
    s.close()


def test_full_uneven_batch_matches_oracle(ctx):
    """The benchmark configuration: 100,000 transforms (N log-uniform over
    2^4..2^10) + 64 x 2^16 + 4 x 2^20, one persistent launch, every job
    bit-exact."""
    b = W.uneven_batch()
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    assert s.engine.status() == bn.OK
    assert np.array_equal(s.output(), s.expected(threads=16))
    s.close()


def test_bounded_wait_reports_timeout_and_context_stays_usable(ctx):
    """Failure path of the persistent kernel without any GPU fault: an injected
    run whose later-pass waits can never be satisfied gives up after a short
    poll limit, the kernel ends, status is BNTT_ETIMEOUT, and the next run on
    the same context is correct."""
    b = W.uneven_batch(seed=10, n_small=200, large=((12, 2),))
    s = Setup(ctx, b)
    jobs = s.jobs()
    bn.check(bn.lib().bntt_batch_inject_wait_timeout(s.engine.handle, 2000))
    s.engine.run_dev(jobs)
    assert s.engine.status() == bn.ETIMEOUT
    assert b"waited too long" in bn.lib().bntt_last_error()
    s.engine.run_dev(jobs)             # next run: no injection, schedule rebuilt
    assert s.engine.status() == bn.OK
    assert np.array_equal(s.output(), s.expected())
    s.close()


def test_several_plans_per_size_scattered_buffers(ctx):
    """Two tables for the same size, jobs in random order at scattered
    (non-contiguous) offsets, several jobs reading the same input into
    different outputs: every output equals the oracle's transform with its
    own plan's table."""
    rng = np.random.default_rng(17)
    spec = [(3, 0), (8, 0), (8, 1), (12, 0), (12, 1), (17, 0)]   # (log2 N, table variant)
    tables = [C.uniform_pairs(5000 + 10 * n + v, 1 << n, C.Q_NTT) for n, v in spec]
    plans = [bn.Plan(ctx, n, C.Q_NTT, C.MU_NTT, t) for (n, _), t in zip(spec, tables)]
    eng = bn.Batch(ctx, plans)
    pick = rng.integers(0, len(spec), size=400)
    pick[:3] = [5, 3, 4]                      # make sure the large plans are used
    sizes = [1 << spec[p][0] for p in pick]
    # inputs: one slot per job, some jobs re-use an earlier job's input
    total_in = sum(sizes) + 4096
    x = C.uniform_pairs(61, total_in, C.Q_NTT)
    dx = DevBuf.from_array(ctx, x)
    in_off, pos = [], 0
    for i, n in enumerate(sizes):
        if i > 10 and rng.random() < 0.1 and sizes[i - 1] == n:
            in_off.append(in_off[-1])         # same input as the previous job
        else:
            pos += int(rng.integers(0, 3))    # gaps between inputs
            in_off.append(pos)
            pos += n
    assert pos <= total_in
    out_total = sum(sizes) * 2
    dy = DevBuf(ctx, out_total * 16)
    out_off, pos = [], 0
    for n in sizes:
        pos += int(rng.integers(0, 5))
        out_off.append(pos)
        pos += n
    assert pos <= out_total
    order = rng.permutation(len(sizes))
    jobs = bn.Batch.jobs([dx.addr + 16 * in_off[i] for i in order],
                         [dy.addr + 16 * out_off[i] for i in order], [int(pick[i]) for i in order])
    eng.run_dev(jobs)
    assert eng.status() == bn.OK
    y = dy.to_array()
    for i in range(len(sizes)):
        p, n = int(pick[i]), sizes[i]
        want = C.oracle_ntt(x[in_off[i]:in_off[i] + n], tables[p], spec[p][0], threads=8, form=1)
        assert np.array_equal(y[out_off[i]:out_off[i] + n], want), f"job {i} (plan {p})"
    dx.free()
    dy.free()
    eng.close()
    for p in plans:
        p.close()


def test_empty_job_list(ctx):
    p = bn.Plan(ctx, 5, C.Q_NTT, C.MU_NTT, C.uniform_pairs(1, 32, C.Q_NTT))
    eng = bn.Batch(ctx, [p])
    before = ctx.launches
    eng.run_dev(bn.Batch.jobs([], [], []))
    assert eng.status() == bn.OK and ctx.launches == before
    eng.close()
    p.close()


def test_inverse_batch_matches_oracle(ctx):
    """bntt_batch_run_inverse_dev: every job of a mix of 2^1..2^10 plus 2^12,
    2^16 and 2^20 equals the oracle's inverse (orc_ntt_inverse_batch) of its
    input, bit for bit."""
    b = W.uneven_batch(seed=31, n_small=2500, small_lo=1, small_hi=10,
                       large=((12, 2), (16, 2), (20, 1)))
    s = Setup(ctx, b)
    s.engine.run_inverse_dev(s.jobs())
    assert s.engine.status() == bn.OK
    got = s.output()
    for i in range(b.count):
        o, logn = int(b.offsets[i]), int(b.logns[i])
        n = 1 << logn
        want = C.oracle_ntt_inverse(s.x[o:o + n], s.tables[logn], logn)
        assert np.array_equal(got[o:o + n], want), f"job {i} (2^{logn})"
    s.close()


def test_forward_then_inverse_batch_round_trip(ctx):
    """Forward batch into y, inverse batch of y back: the inputs return, for
    the uneven mix with large transforms (both directions one launch)."""
    b = W.uneven_batch(seed=32, n_small=5000, large=((16, 4), (20, 2)))
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    zs = DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    back = bn.Batch.jobs([s.dy.addr + o for o in offs], [zs.addr + o for o in offs],
                         [s.plan_ids[int(n)] for n in b.logns])
    s.engine.run_inverse_dev(back)
    assert s.engine.status() == bn.OK
    assert np.array_equal(zs.to_array(), s.x)
    assert s.engine.last_launches == 2   # schedule build on the device, then the persistent kernel
    zs.free()
    s.close()


def test_inverse_batch_rejects_slow_modulus():
    q = (1 << 123) + 12345678901
    c = bn.Context(0)
    p = bn.Plan(c, 5, q, (1 << 251) // q, C.uniform_pairs(1, 32, q))
    eng = bn.Batch(c, [p])
    d = DevBuf(c, 32 * 16)
    with pytest.raises(bn.BnttError) as e:
        eng.run_inverse_dev(bn.Batch.jobs([d.addr], [d.addr], [0]))
    assert e.value.status == bn.EINVAL
    d.free()
    eng.close()
    p.close()
    c.close()


def test_every_large_split_in_one_batch(ctx):
    """Large sizes whose engine splits end in a 3- or 5-stage pass or need
    three passes (2^11 = 8+3, 2^13 = 8+5, 2^17 = 6+8+3, 2^19 = 8+8+3,
    2^21 = 8+8+5) in one mixed launch: bit-exact against the oracle up to
    2^17, and forward-then-inverse round trips for all."""
    b = W.uneven_batch(seed=33, n_small=300, large=((11, 2), (13, 1), (17, 1), (19, 1), (21, 1)))
    s = Setup(ctx, b)
    s.engine.run_dev(s.jobs())
    assert s.engine.status() == bn.OK
    y = s.output()
    for i in range(b.count):
        o, logn = int(b.offsets[i]), int(b.logns[i])
        if 11 <= logn <= 17:
            n = 1 << logn
            want = C.oracle_ntt(s.x[o:o + n], s.tables[logn], logn, form=1)
            assert np.array_equal(y[o:o + n], want), f"job {i} (2^{logn})"
    zs = DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    back = bn.Batch.jobs([s.dy.addr + o for o in offs], [zs.addr + o for o in offs],
                         [s.plan_ids[int(n)] for n in b.logns])
    s.engine.run_inverse_dev(back)
    assert s.engine.status() == bn.OK
    assert np.array_equal(zs.to_array(), s.x)
    zs.free()
    s.close()


def test_run_host_reports_timeout_and_recovers(ctx):
    """The host-buffer pipeline's failure path: an injected run whose waits
    can never be satisfied returns BNTT_ETIMEOUT from bntt_batch_run_host
    itself (every group's error word is read), and the next run is correct."""
    b = W.uneven_batch(seed=12, n_small=300, large=((12, 2), (16, 1)))
    s = Setup(ctx, b)
    y = np.zeros_like(s.x)
    xs = [s.x.ctypes.data + 16 * int(o) for o in b.offsets]
    ys = [y.ctypes.data + 16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs(xs, ys, [s.plan_ids[int(n)] for n in b.logns])
    bn.check(bn.lib().bntt_batch_inject_wait_timeout(s.engine.handle, 2000))
    with pytest.raises(bn.BnttError) as e:
        s.engine.run_host(jobs)
    assert e.value.status == bn.ETIMEOUT
    s.engine.run_host(jobs)
    assert np.array_equal(y, s.expected())
    s.engine.run_host(jobs)             # cached schedules
    assert np.array_equal(y, s.expected())
    s.close()


def test_run_host_async_chained_in_place(ctx):
    """Back-to-back asynchronous host runs are ordered group by group: with
    in-place jobs (x == y on the host) three queued runs give ntt(ntt(ntt(x)))
    for every job, which holds only if each run's input copy of a group waits
    for the previous run's output copy of it."""
    b = W.uneven_batch(seed=13, n_small=2000, large=((16, 3), (20, 1)))
    s = Setup(ctx, b)
    buf = s.x.copy()
    ptrs = [buf.ctypes.data + 16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs(ptrs, ptrs, [s.plan_ids[int(n)] for n in b.logns])
    for _ in range(3):
        s.engine.run_host_async(jobs)
    s.engine.sync()
    ns = [int(n) for n in b.logns]
    ts = [s.tables[n] for n in ns]
    want = [s.x[o:o + (1 << n)] for o, n in zip(b.offsets, ns)]
    for _ in range(3):
        want = C.oracle_ntt_jobs(want, ts, ns, threads=8)
    assert np.array_equal(buf, np.concatenate(want))
    s.close()


def test_run_host_async_reports_timeout_at_sync(ctx):
    """An injected wait timeout in a queued host run is reported by
    bntt_batch_sync, also when a later run with another job list had to
    rebuild the schedules first; the runs after it are correct."""
    b = W.uneven_batch(seed=14, n_small=300, large=((12, 2), (16, 1)))
    s = Setup(ctx, b)
    y = np.zeros_like(s.x)
    xs = [s.x.ctypes.data + 16 * int(o) for o in b.offsets]
    ys = [y.ctypes.data + 16 * int(o) for o in b.offsets]
    ids = [s.plan_ids[int(n)] for n in b.logns]
    jobs = bn.Batch.jobs(xs, ys, ids)
    part = bn.Batch.jobs(xs[:100], ys[:100], ids[:100])
    bn.check(bn.lib().bntt_batch_inject_wait_timeout(s.engine.handle, 2000))
    s.engine.run_host_async(jobs)
    s.engine.run_host_async(part)        # another job list: rebuild after the faulty run
    with pytest.raises(bn.BnttError) as e:
        s.engine.sync()
    assert e.value.status == bn.ETIMEOUT
    s.engine.sync()                       # reported once
    s.engine.run_host_async(jobs)
    s.engine.run_host_async(jobs)
    s.engine.sync()
    assert np.array_equal(y, s.expected())
    s.close()


def test_alternating_job_lists_without_sync(ctx):
    """Two job lists (different sizes and outputs) queued in turn, with no
    synchronisation in between: each new list is copied into the schedule
    buffer the running launch does not read and launched directly; a list
    seen again is replayed from its graph.  Both outputs equal the oracle."""
    b = W.uneven_batch(seed=15, n_small=3000, large=((16, 2), (20, 1)))
    s = Setup(ctx, b)
    ya = DevBuf(ctx, b.total * 16)
    yb = DevBuf(ctx, b.total * 16)
    ids = [s.plan_ids[int(n)] for n in b.logns]
    xs = [s.dx.addr + 16 * int(o) for o in b.offsets]
    ja = bn.Batch.jobs(xs, [ya.addr + 16 * int(o) for o in b.offsets], ids)
    half = b.count // 2
    jb = bn.Batch.jobs(xs[half:][::-1], [yb.addr + 16 * int(o) for o in b.offsets[half:]][::-1], ids[half:][::-1])
    for _ in range(3):
        s.engine.run_dev(ja)
        s.engine.run_dev(jb)
    s.engine.run_dev(ja)
    s.engine.run_dev(ja)             # the same list again: graph replay
    assert s.engine.status() == bn.OK
    want = s.expected()
    assert np.array_equal(ya.to_array(b.total), want)
    o = int(b.offsets[half])
    assert np.array_equal(yb.to_array(b.total)[o:], want[o:])
    ya.free()
    yb.free()
    s.close()

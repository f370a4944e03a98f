"""The serving loop (bntt_server_*): continuous batching of mixed requests.

Every result must be bit-identical alone and in the mix (integer results:
tolerance 0) and equal to the oracle; admission respects the HBM budget;
trace replays in both modes complete every request."""
import ctypes

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
NTT_SIZES = [4, 5, 8, 10, 12, 16]


class Fixture:
    def __init__(self, budget=0, slots=0, max_batch=0):
        self.ctx = bn.Context(0)
        self.tables = {n: C.uniform_pairs(W.SEED_TWIDDLE_BASE + n, 1 << n, C.Q_NTT) for n in NTT_SIZES}
        self.plans = [bn.Plan(self.ctx, n, C.Q_NTT, C.MU_NTT, self.tables[n]) for n in NTT_SIZES]
        self.srv = bn.Server(self.ctx, self.plans, C.Q_BLAS, C.MU_BLAS, hbm_budget=budget,
                             slots=slots, max_batch=max_batch)
        self.bufs = []

    def dev(self, arr):
        d = DevBuf.from_array(self.ctx, arr)
        self.bufs.append(d)
        return d

    def close(self):
        self.srv.close()
        for d in self.bufs:
            d.free()
        for p in self.plans:
            p.close()
        self.ctx.close()


def make_requests(fx, count, seed):
    """Random mix: 70% NTTs over NTT_SIZES, 30% vvmul / axpy of 2^10..2^16."""
    rng = np.random.default_rng(seed)
    reqs, expect = [], []
    for i in range(count):
        if rng.random() < 0.7:
            pi = int(rng.integers(len(NTT_SIZES)))
            n = NTT_SIZES[pi]
            x = C.uniform_pairs(1000 * seed + i, 1 << n, C.Q_NTT)
            d = fx.dev(x)
            r = bn.RequestC(bn.REQ_NTT, pi, 0, d.addr, None, bn.U128.of(0), i, 0.0)
            expect.append(("ntt", n, x, None, 0))
        else:
            ln = 1 << int(rng.integers(10, 17))
            a = C.uniform_pairs(2000 * seed + i, ln, C.Q_BLAS)
            b = C.uniform_pairs(3000 * seed + i, ln, C.Q_BLAS)
            kind = bn.REQ_VVMUL if rng.random() < 0.5 else bn.REQ_AXPY
            xs = int(C.from_pairs(C.uniform_pairs(4000 * seed + i, 1, C.Q_BLAS))[0])
            da, db = fx.dev(a), fx.dev(b)
            r = bn.RequestC(kind, 0, ln, da.addr, db.addr, bn.U128.of(xs), i, 0.0)
            expect.append(("vvmul" if kind == bn.REQ_VVMUL else "axpy", ln, a, b, xs))
        reqs.append(r)
    return reqs, expect


def oracle_of(fx, e):
    kind, n, a, b, xs = e
    if kind == "ntt":
        return C.oracle_ntt(a, fx.tables[n], n)
    return C.oracle_blas(kind, a, b, C.Q_BLAS, C.MU_BLAS, xs)


def fetch(fx, cpl):
    out = np.empty((cpl.bytes // 16, 2), dtype=np.uint64)
    fx.ctx.synchronize()
    bn.check(bn.lib().bntt_copy_d2h(fx.ctx.handle, out.ctypes.data, cpl.y, cpl.bytes))
    return out


def run_mix(fx, reqs):
    for r in reqs:
        fx.srv.submit(r)
    fx.srv.drain()
    outs = {}
    for cpl in fx.srv.poll(len(reqs) + 10):
        assert cpl.status == bn.OK
        outs[cpl.tag] = fetch(fx, cpl)
        fx.srv.release(cpl.y)
    return outs


def test_mix_equals_alone_and_oracle():
    fx = Fixture()
    reqs, expect = make_requests(fx, 120, seed=1)
    mixed = run_mix(fx, reqs)
    assert len(mixed) == len(reqs)
    for i, r in enumerate(reqs):
        alone = run_mix(fx, [r])[i]
        assert np.array_equal(mixed[i], alone), f"request {i} differs alone vs in the mix"
        assert np.array_equal(mixed[i], oracle_of(fx, expect[i])), f"request {i} differs from the oracle"
    st = fx.srv.stats()
    assert st["completed"] == st["submitted"] == 240
    fx.close()


def test_admission_waits_for_budget():
    # 4 MiB arena: 2^16-point NTT outputs (1 MiB each) admit at most 4 at once
    fx = Fixture(budget=4 << 20, slots=4)
    n = 16
    pi = NTT_SIZES.index(n)
    xs = [C.uniform_pairs(500 + i, 1 << n, C.Q_NTT) for i in range(12)]
    reqs = [bn.RequestC(bn.REQ_NTT, pi, 0, fx.dev(x).addr, None, bn.U128.of(0), i, 0.0)
            for i, x in enumerate(xs)]
    outs = {}
    for r in reqs:
        fx.srv.submit(r)
    while len(outs) < len(reqs):      # release as results arrive, freeing the arena
        for cpl in fx.srv.poll():
            outs[cpl.tag] = fetch(fx, cpl)
            fx.srv.release(cpl.y)
    for i, x in enumerate(xs):
        assert np.array_equal(outs[i], C.oracle_ntt(x, fx.tables[n], n, form=1))
    st = fx.srv.stats()
    assert st["peak_bytes"] <= 4 << 20
    assert st["admission_waits"] > 0
    big = bn.RequestC(bn.REQ_VVMUL, 0, 1 << 20, reqs[0].x, reqs[0].x, bn.U128.of(0), 99, 0.0)
    rc = bn.lib().bntt_server_submit(fx.srv.handle, ctypes.byref(big))
    assert rc == bn.EBUDGET
    fx.close()


@pytest.mark.parametrize("serial", [False, True])
def test_replay_completes_every_request(serial):
    fx = Fixture()
    reqs, _ = make_requests(fx, 200, seed=3)
    gaps = np.random.default_rng(0).exponential(1 / 50_000, size=len(reqs))
    arr = (bn.RequestC * len(reqs))(*reqs)
    t = 0.0
    for i in range(len(reqs)):
        arr[i].t_arrive = t
        t += gaps[i]
    lat, wall = fx.srv.replay(arr, serial=serial)
    assert np.all(lat > 0) and np.all(np.isfinite(lat))
    assert wall >= arr[len(reqs) - 1].t_arrive
    fx.close()


def test_launch_output_cap():
    # one launch admits at most 256 MiB of outputs: six 128 MiB vvmuls take at
    # least three launches; a 512 MiB request larger than the cap runs alone
    fx = Fixture(slots=1)
    ln = 1 << 23
    a = C.uniform_pairs(71, ln, C.Q_BLAS)
    b = C.uniform_pairs(72, ln, C.Q_BLAS)
    da, db = fx.dev(a), fx.dev(b)
    big = np.concatenate([a, a, a, a])
    bigb = np.concatenate([b, b, b, b])
    dba, dbb = fx.dev(big), fx.dev(bigb)
    reqs = [bn.RequestC(bn.REQ_VVMUL, 0, ln, da.addr, db.addr, bn.U128.of(0), i, 0.0) for i in range(6)]
    reqs.append(bn.RequestC(bn.REQ_VVMUL, 0, 4 * ln, dba.addr, dbb.addr, bn.U128.of(0), 6, 0.0))
    outs = run_mix(fx, reqs)
    head = 1 << 12
    want = C.oracle_blas("vvmul", a[:head], b[:head], C.Q_BLAS, C.MU_BLAS, 0)
    for i in range(6):
        assert np.array_equal(outs[i], outs[0])
    assert np.array_equal(outs[0][:head], want)
    assert np.array_equal(outs[6][3 * ln:3 * ln + head], want)
    st = fx.srv.stats()
    assert st["launches"] >= 4
    assert st["completed"] == 7
    fx.close()


def test_other_batches_do_not_break_server_launches():
    """A batch of only the tiniest transforms (one-thread tiles, the least
    shared memory) runs between server launches: the server's later launches
    of 2^10-point tiles still run and are correct (no shared-memory limit of
    the common kernel is set per job list)."""
    fx = Fixture(slots=1)
    tiny_t = C.uniform_pairs(61, 2, C.Q_NTT)
    tiny_plan = bn.Plan(fx.ctx, 1, C.Q_NTT, C.MU_NTT, tiny_t)
    tiny_engine = bn.Batch(fx.ctx, [tiny_plan])
    xt = C.uniform_pairs(62, 2 * 64, C.Q_NTT)
    dxt, dyt = fx.dev(xt), fx.dev(np.zeros_like(xt))
    jobs = bn.Batch.jobs([dxt.addr + 32 * i for i in range(64)], [dyt.addr + 32 * i for i in range(64)], [0] * 64)
    n = 10
    pi = NTT_SIZES.index(n)
    x = C.uniform_pairs(63, 1 << n, C.Q_NTT)
    r = bn.RequestC(bn.REQ_NTT, pi, 0, fx.dev(x).addr, None, bn.U128.of(0), 0, 0.0)
    run_mix(fx, [r])
    tiny_engine.run_dev(jobs)
    assert tiny_engine.status() == bn.OK
    out = run_mix(fx, [r])
    assert np.array_equal(out[0], C.oracle_ntt(x, fx.tables[n], n))
    assert np.array_equal(dyt.to_array(128), C.oracle_ntt(xt, tiny_t, 1))
    tiny_engine.close()
    tiny_plan.close()
    fx.close()

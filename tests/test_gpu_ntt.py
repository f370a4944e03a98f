"""GPU parity of the forward NTT (src/ntt_scalar.c:582-627), bit-exact.

Covers the reference's golden vectors (N = 16..1024), fixtures produced by the
compiled reference for N = 4..2^20 (full outputs up to 2^12, SHA-256 above),
boundary inputs, uniform batches against the oracle, both buffer layouts,
both arithmetic policies, other moduli, in-place calls and argument errors.
"""
import ctypes
import hashlib

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from gpu_util import DevBuf, hilo_to_u128, u128_to_hilo

pytestmark = pytest.mark.gpu

GOLD = C.load_golden()
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def ctx():
    c = bn.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx_ref():
    c = bn.Context(0, arith=bn.ARITH_REFERENCE)
    yield c
    c.close()


def run_dev(ctx, x, t, logn, q=C.Q_NTT, mu=C.MU_NTT, layout=bn.LAYOUT_HILO, inplace=False):
    plan = bn.Plan(ctx, logn, q, mu, t, layout)
    dx = DevBuf.from_array(ctx, x)
    dy = dx if inplace else DevBuf(ctx, x.nbytes)
    bn.check(bn.lib().bntt_ntt_forward_dev(plan.handle, dy.ptr, dx.ptr, x.shape[0] >> logn))
    y = dy.to_array(x.shape[0])
    dx.free()
    if not inplace:
        dy.free()
    plan.close()
    return y


@pytest.mark.parametrize("logn", range(4, 11))
@pytest.mark.parametrize("which", ["auto", "reference"])
def test_reference_goldens_dev(ctx, ctx_ref, logn, which):
    n = 1 << logn
    y = run_dev(ctx if which == "auto" else ctx_ref, GOLD[f"x_{n}"], GOLD[f"twd_{n}"], logn)
    assert np.array_equal(y, GOLD[f"ver_{n}"])


@pytest.mark.parametrize("logn", range(4, 11))
def test_reference_goldens_host(ctx, logn):
    n = 1 << logn
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, GOLD[f"twd_{n}"])
    y = np.empty((n, 2), dtype=np.uint64)
    plan.forward(y, GOLD[f"x_{n}"])
    assert np.array_equal(y, GOLD[f"ver_{n}"])


def test_reference_shaped_ntt_call():
    y = np.empty((1024, 2), dtype=np.uint64)
    bn.ntt(y, GOLD["x_1024"], C.Q_NTT, C.MU_NTT, GOLD["twd_1024"])
    assert np.array_equal(y, GOLD["ver_1024"])


@pytest.mark.parametrize("logn", range(2, 21))
def test_reference_generated(ctx, logn):
    n = 1 << logn
    x = C.uniform_pairs(1000 + logn, n, C.Q_NTT)
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    y = run_dev(ctx, x, t, logn)
    if logn <= 12:
        assert np.array_equal(y, GEN[f"ntt_y_{logn}"])
    assert sha(y) == str(GEN[f"ntt_sha_{logn}"])


@pytest.mark.parametrize("logn", [13, 16, 20])
def test_reference_generated_arith_reference(ctx_ref, logn):
    n = 1 << logn
    x = C.uniform_pairs(1000 + logn, n, C.Q_NTT)
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    assert sha(run_dev(ctx_ref, x, t, logn)) == str(GEN[f"ntt_sha_{logn}"])


@pytest.mark.parametrize("logn", [4, 7, 10])
@pytest.mark.parametrize("edge", ["zero", "one", "qm1", "q", "two64", "tqm1"])
def test_edge_inputs(ctx, logn, edge):
    n = 1 << logn
    q = C.Q_NTT
    x = C.uniform_pairs(1000 + logn, n, q)
    t = C.uniform_pairs(2000 + logn, n, q)
    vals = {"zero": 0, "one": 1, "qm1": q - 1, "q": q, "two64": 1 << 64}
    if edge == "tqm1":
        t = C.to_pairs([q - 1] * n)
    else:
        x = C.to_pairs([vals[edge]] * n)
    assert np.array_equal(run_dev(ctx, x, t, logn), GEN[f"edge_{edge}_{logn}"])


@pytest.mark.parametrize("logn,batch", [(1, 7), (3, 1000), (4, 4099), (5, 333), (6, 1000),
                                        (7, 513), (8, 300), (9, 129), (10, 130), (11, 9),
                                        (12, 5), (14, 3), (15, 2), (16, 2), (19, 1)])
def test_uniform_batch_matches_oracle(ctx, logn, batch):
    n = 1 << logn
    x = C.uniform_pairs(7 + logn, n * batch, C.Q_NTT)
    t = C.uniform_pairs(8 + logn, n, C.Q_NTT)
    y = run_dev(ctx, x, t, logn)
    assert np.array_equal(y, C.oracle_ntt(x, t, logn, threads=8, form=1))


@pytest.mark.parametrize("logn", [4, 7, 10, 12, 16])
def test_layout_u128(ctx, logn):
    n = 1 << logn
    x = C.uniform_pairs(61, n * 3, C.Q_NTT)
    t = C.uniform_pairs(62, n, C.Q_NTT)
    y = run_dev(ctx, hilo_to_u128(x), hilo_to_u128(t), logn, layout=bn.LAYOUT_U128)
    assert np.array_equal(u128_to_hilo(y), C.oracle_ntt(x, t, logn, threads=8))


@pytest.mark.parametrize("logn", [5, 10, 13])
def test_in_place(ctx, logn):
    n = 1 << logn
    x = C.uniform_pairs(71, n * 2, C.Q_NTT)
    t = C.uniform_pairs(72, n, C.Q_NTT)
    assert np.array_equal(run_dev(ctx, x, t, logn, inplace=True), C.oracle_ntt(x, t, logn))


@pytest.mark.parametrize("q", [(1 << 124) - 3, (1 << 124) - 0x7bfffff, (1 << 124) - ((1 << 31) - 1),
                               (1 << 123) + 12345678901, (1 << 127) + 99])
@pytest.mark.parametrize("logn", [4, 10, 12])
def test_other_moduli(ctx, q, logn):
    mu = ((1 << 251) // q) & ((1 << 128) - 1)
    n = 1 << logn
    x = C.uniform_pairs(81, n * 2, q)
    t = C.uniform_pairs(82, n, q)
    assert np.array_equal(run_dev(ctx, x, t, logn, q, mu), C.oracle_ntt(x, t, logn, q, mu))


def test_full_range_inputs_reference_arith(ctx_ref):
    """Out-of-domain 128-bit inputs: the replica arithmetic still matches."""
    rng = np.random.default_rng(5)
    for logn in (4, 9, 11):
        n = 1 << logn
        x = rng.integers(0, 2**64, size=(2 * n, 2), dtype=np.uint64)
        t = rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)
        assert np.array_equal(run_dev(ctx_ref, x, t, logn), C.oracle_ntt(x, t, logn))


def test_host_pipeline_many_chunks(ctx):
    """bntt_ntt_forward_host splits large batches into pipelined chunks."""
    logn = 10
    n = 1 << logn
    batch = 5000  # > 2 chunks of 32 MiB
    x = C.uniform_pairs(91, n * batch, C.Q_NTT)
    t = C.uniform_pairs(92, n, C.Q_NTT)
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = np.empty_like(x)
    plan.forward(y, x)
    assert np.array_equal(y, C.oracle_ntt(x, t, logn, threads=8, form=1))


def test_invalid_arguments(ctx):
    L = bn.lib()
    m = bn.modulus(C.Q_NTT, C.MU_NTT)
    t = C.uniform_pairs(1, 1024, C.Q_NTT)
    h = ctypes.c_void_p()
    assert L.bntt_plan_create(ctx.handle, ctypes.byref(h), 0, ctypes.byref(m), t.ctypes.data, 0) == bn.EINVAL
    assert L.bntt_plan_create(ctx.handle, ctypes.byref(h), 25, ctypes.byref(m), t.ctypes.data, 0) == bn.EINVAL
    assert L.bntt_plan_create(ctx.handle, ctypes.byref(h), 10, ctypes.byref(m), None, 0) == bn.EINVAL
    plan = bn.Plan(ctx, 10, C.Q_NTT, C.MU_NTT, t)
    d = DevBuf(ctx, 1024 * 16 + 16)
    assert L.bntt_ntt_forward_dev(plan.handle, d.addr + 8, d.ptr, 1) == bn.EINVAL
    assert L.bntt_ntt_forward_dev(plan.handle, None, None, 0) == bn.OK  # empty batch
    d.free()
    plan.close()


def test_budget_rejects_plan(ctx):
    c = bn.Context(0)
    c.set_hbm_budget(1024)
    with pytest.raises(bn.BnttError) as e:
        bn.Plan(c, 10, C.Q_NTT, C.MU_NTT, C.uniform_pairs(1, 1024, C.Q_NTT))
    assert e.value.status == bn.EBUDGET
    c.close()


def rare_sum_inputs(logn, batch, q=C.Q_NTT):
    """Transforms whose stage-0 pairs (j, j + N/2) sum to addmod's rare cases
    under an all-ones table: sums in (q, 2^124), sums equal to q and 2^124,
    sums above 2^124 whose low 64 bits equal q's (the borrow quirk), other
    sums with limb 1 = 0xFFFFFFFF, and ordinary sums.  Each sum s is split as
    x = s - s // 2, y = s // 2, both at most q."""
    k = (1 << 124) - q
    rng = np.random.default_rng(logn)
    sums = [q + 1, q + 2, q + k - 1, q, q - 1, 1 << 124, (1 << 124) + 1, (1 << 124) - 1]
    sums += [q + j * (1 << 64) for j in (1, 2, 3, 1 << 40, (q >> 64) - 1)]
    for _ in range(24):
        hi = int(rng.integers(0, 1 << 61)) % (q >> 64)
        lo = (0xFFFFFFFF << 32) | int(rng.integers(0, 1 << 32))
        s = (hi << 64) | lo
        sums.append(s if s < 2 * q else s - q)
    sums += [int(v) for v in C.from_pairs(C.uniform_pairs(77 + logn, 32, 2 * q))]
    half = 1 << (logn - 1)
    xs = np.empty((batch << logn, 2), dtype=np.uint64)
    for t in range(batch):
        lo_half, hi_half = [], []
        for i in range(half):
            s = sums[(t * half + i) % len(sums)]
            hi_half.append(s // 2)
            lo_half.append(s - s // 2)
        xs[t << logn:(t + 1) << logn] = C.to_pairs(lo_half + hi_half)
    return xs


@pytest.mark.parametrize("logn,batch", [(1, 70), (4, 9), (10, 2), (12, 1), (16, 1)])
def test_addmod_rare_sums(ctx, logn, batch):
    """The fast addmod's exceptional sums (one in 2^32 for uniform data, so
    constructed here) through the plan kernels and the persistent batch
    kernel, against the oracle."""
    n = 1 << logn
    x = rare_sum_inputs(logn, batch)
    t = C.to_pairs([1] * n)
    want = C.oracle_ntt(x, t, logn)
    assert np.array_equal(run_dev(ctx, x, t, logn), want)
    plan = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    engine = bn.Batch(ctx, [plan])
    dx = DevBuf.from_array(ctx, x)
    dy = DevBuf(ctx, x.nbytes)
    jobs = bn.Batch.jobs([dx.addr + 16 * n * i for i in range(batch)],
                         [dy.addr + 16 * n * i for i in range(batch)], [0] * batch)
    engine.run_dev(jobs)
    assert engine.status() == bn.OK
    assert np.array_equal(dy.to_array(x.shape[0]), want)
    dx.free()
    dy.free()
    engine.close()
    plan.close()

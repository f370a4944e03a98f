"""GPU parity of the NTT-friendly prime mode.

Plans built with bntt_plan_create_negacyclic generate the root-power table
T[k] = psi^brv(k) on the device; their transforms must equal the compiled
reference ntt() (src/ntt_scalar.c:582) run with the same prime, mu and a table
built in pure Python (fixtures nc_* in tests/golden/ref_gen.npz), bit for bit.
At 2^20 the convolution theorem with a monomial is checked as a
size-independent property as well.
"""
import hashlib

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from benchntt_b200 import workloads as W
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")
Q_NC = C.from_pairs(GEN["nc_q"])[0]
MU_NC = (1 << 251) // Q_NC
ROOT21 = C.from_pairs(GEN["nc_root21"])[0]


def psi_for(logn):
    return pow(ROOT21, 1 << (C.NC_LOG2_ORDER - logn - 1), Q_NC)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.fixture(scope="module")
def ctx():
    c = bn.Context(0)
    yield c
    c.close()


def dev_forward(ctx, plan, x):
    dx = DevBuf.from_array(ctx, x)
    dy = DevBuf(ctx, x.nbytes)
    bn.check(bn.lib().bntt_ntt_forward_dev(plan.handle, dy.ptr, dx.ptr, x.shape[0] >> plan.log2n))
    y = dy.to_array()
    dx.free()
    dy.free()
    return y


@pytest.mark.parametrize("logn", range(2, 21))
def test_device_table_plan_matches_reference(ctx, logn):
    x = C.uniform_pairs(1000 + logn, 1 << logn, Q_NC)
    p = bn.Plan.negacyclic(ctx, logn, Q_NC, MU_NC, psi_for(logn))
    y = dev_forward(ctx, p, x)
    if logn <= 12:
        assert np.array_equal(y, GEN[f"nc_y_{logn}"])
    assert sha(y) == str(GEN[f"nc_sha_{logn}"])
    p.close()


@pytest.mark.parametrize("logn", [3, 10, 16])
def test_device_table_equals_host_table(ctx, logn):
    """The table generated on the device and the host table give the same
    transform of a batch (and the host table equals the pure-Python one)."""
    psi = psi_for(logn)
    t_host = bn.twiddles_negacyclic(Q_NC, MU_NC, logn, psi)
    assert np.array_equal(t_host, C.negacyclic_table(Q_NC, logn, psi))
    x = C.uniform_pairs(55, 8 << logn, Q_NC)
    p_dev = bn.Plan.negacyclic(ctx, logn, Q_NC, MU_NC, psi)
    p_host = bn.Plan(ctx, logn, Q_NC, MU_NC, t_host)
    y = dev_forward(ctx, p_dev, x)
    assert np.array_equal(y, dev_forward(ctx, p_host, x))
    assert np.array_equal(y, C.oracle_ntt(x, t_host, logn, Q_NC, MU_NC, form=1, threads=8))
    p_dev.close()
    p_host.close()


@pytest.mark.parametrize("logn", [4, 10, 12])
def test_negacyclic_dft_definition_small(ctx, logn):
    """A few outputs against Y[i] = sum_j X[j] psi^((2 brv(i) + 1) j)."""
    n = 1 << logn
    psi = psi_for(logn)
    x = C.uniform_pairs(66, n, Q_NC)
    y = C.from_pairs(dev_forward(ctx, bn.Plan.negacyclic(ctx, logn, Q_NC, MU_NC, psi), x))
    xs = C.from_pairs(x)
    for i in (0, 1, n // 3, n - 1):
        r = pow(psi, 2 * C.brv(i, logn) + 1, Q_NC)
        assert y[i] == sum(xj * pow(r, j, Q_NC) for j, xj in enumerate(xs)) % Q_NC


@pytest.mark.parametrize("logn,shift", [(16, 12345), (20, 777777)])
def test_monomial_convolution_at_full_size(ctx, logn, shift):
    """NTT(a * x^s mod (x^N + 1)) = NTT(a) o NTT(x^s) at 2^16 and 2^20: the
    negacyclic shift moves a_j to j + s and negates what wraps.  All three
    transforms run on the device; the pointwise product is the oracle's."""
    n = 1 << logn
    p = bn.Plan.negacyclic(ctx, logn, Q_NC, MU_NC, psi_for(logn))
    a = C.uniform_pairs(99, n, Q_NC)
    vals = np.array(C.from_pairs(a), dtype=object)
    shifted = np.roll(vals, shift)
    shifted[:shift] = [(Q_NC - v) % Q_NC for v in shifted[:shift]]
    mono = np.zeros((n, 2), dtype=np.uint64)
    mono[shift] = C.to_pairs([1])[0]
    lhs = dev_forward(ctx, p, C.to_pairs(list(shifted)))
    rhs = C.oracle_blas("vvmul", dev_forward(ctx, p, a), dev_forward(ctx, p, mono), Q_NC, MU_NC)
    assert np.array_equal(lhs, rhs)
    p.close()


def test_mixed_batch_of_negacyclic_plans(ctx):
    """The persistent kernel over root-power plans of every size 2^4..2^10 plus
    2^16 and 2^20 jobs, bit-exact against the oracle job by job."""
    b = W.uneven_batch(seed=12, n_small=3000, large=((16, 2), (20, 1)))
    plans = {n: bn.Plan.negacyclic(ctx, n, Q_NC, MU_NC, psi_for(n)) for n in b.sizes}
    tables = {n: C.negacyclic_table(Q_NC, n, psi_for(n)) for n in b.sizes}
    pid = {n: i for i, n in enumerate(b.sizes)}
    eng = bn.Batch(ctx, [plans[n] for n in b.sizes])
    x = C.uniform_pairs(W.SEED_INPUT, b.total, Q_NC)
    dx, dy = DevBuf.from_array(ctx, x), DevBuf(ctx, b.total * 16)
    offs = [16 * int(o) for o in b.offsets]
    jobs = bn.Batch.jobs([dx.addr + o for o in offs], [dy.addr + o for o in offs],
                         [pid[int(n)] for n in b.logns])
    eng.run_dev(jobs)
    assert eng.status() == bn.OK
    xs = [x[o:o + (1 << n)] for o, n in zip(b.offsets, b.logns)]
    want = np.concatenate(C.oracle_ntt_jobs(xs, [tables[int(n)] for n in b.logns],
                                            [int(n) for n in b.logns], Q_NC, MU_NC, threads=16))
    assert np.array_equal(dy.to_array(), want)
    dx.free()
    dy.free()
    eng.close()
    for p in plans.values():
        p.close()


def test_plan_rejects_bad_root_and_slow_modulus(ctx):
    with pytest.raises(bn.BnttError):
        bn.Plan.negacyclic(ctx, 10, Q_NC, MU_NC, psi_for(9))        # order 2^10, not 2^11
    q = (1 << 123) + 12345678901                                      # not pseudo-Mersenne
    with pytest.raises(bn.BnttError):
        bn.Plan.negacyclic(ctx, 4, q, (1 << 251) // q, 1)

"""GPU parity of the inverse transform (bntt_ntt_inverse_dev).

The reference has no inverse; the oracle's restatement (orc_ntt_inverse_batch
in oracle/bntt_oracle.c) is the checker, bit for bit (integer results,
tolerance 0).  Size-independent properties back it at every size up to 2^20:
ntt^-1(ntt(x)) = x, the reference's own golden outputs invert to its inputs,
and in the friendly-prime mode ntt^-1(ntt(a) o ntt(b)) is the negacyclic
product a * b mod (x^N + 1).
"""
import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
GOLD = C.load_golden()
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")
Q_NC = C.from_pairs(GEN["nc_q"])[0]
MU_NC = (1 << 251) // Q_NC
ROOT21 = C.from_pairs(GEN["nc_root21"])[0]


@pytest.fixture(scope="module")
def ctx():
    c = bn.Context(0)
    yield c
    c.close()


def dev_call(ctx, plan, fn, a, inplace=False):
    da = DevBuf.from_array(ctx, a)
    db = da if inplace else DevBuf(ctx, a.nbytes)
    bn.check(fn(plan.handle, db.ptr, da.ptr, a.shape[0] >> plan.log2n))
    out = db.to_array()
    da.free()
    if not inplace:
        db.free()
    return out


def inverse(ctx, plan, y, inplace=False):
    return dev_call(ctx, plan, bn.lib().bntt_ntt_inverse_dev, y, inplace)


def forward(ctx, plan, x):
    return dev_call(ctx, plan, bn.lib().bntt_ntt_forward_dev, x)


@pytest.mark.parametrize("logn,batch", [(1, 9), (2, 5), (3, 300), (4, 33), (5, 70), (6, 40), (7, 20),
                                        (8, 9), (9, 8), (10, 16), (10, 1500), (11, 4), (12, 2), (13, 1)])
def test_inverse_matches_oracle(ctx, logn, batch):
    n = 1 << logn
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    y = C.uniform_pairs(7000 + logn, batch * n, C.Q_NTT)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    assert np.array_equal(inverse(ctx, p, y), C.oracle_ntt_inverse(y, t, logn))
    p.close()


@pytest.mark.parametrize("logn", range(4, 11))
def test_reference_goldens_invert_to_inputs(ctx, logn):
    n = 1 << logn
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, GOLD[f"twd_{n}"])
    assert np.array_equal(inverse(ctx, p, GOLD[f"ver_{n}"]), GOLD[f"x_{n}"])
    p.close()


@pytest.mark.parametrize("logn,batch", [(5, 64), (14, 4), (16, 2), (18, 1), (20, 2)])
def test_round_trip_all_sizes(ctx, logn, batch):
    """ntt^-1(ntt(x)) = x through one to three HBM passes each way; at 2^16 the
    inverse also equals the oracle's."""
    n = 1 << logn
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    x = C.uniform_pairs(9000 + logn, batch * n, C.Q_NTT)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = forward(ctx, p, x)
    assert np.array_equal(inverse(ctx, p, y), x)
    if logn == 16:
        assert np.array_equal(inverse(ctx, p, y), C.oracle_ntt_inverse(y, t, logn))
    p.close()


@pytest.mark.parametrize("logn", [15, 19, 21, 22, 23, 24])
def test_round_trip_every_split(ctx, logn):
    """ntt^-1(ntt(x)) = x for the sizes whose pass splits the other tests do
    not reach: strided passes of 6 and 7 stages, contiguous last passes of
    8 and 10 stages, up to 2^24 points (one transform)."""
    n = 1 << logn
    t = C.uniform_pairs(3000 + logn, n, C.Q_NTT)
    x = C.uniform_pairs(4000 + logn, n, C.Q_NTT)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = forward(ctx, p, x)
    assert not np.array_equal(y, x)
    assert np.array_equal(inverse(ctx, p, y), x)
    p.close()


@pytest.mark.parametrize("logn", [10, 12])
def test_in_place_and_u128_layout(ctx, logn):
    n = 1 << logn
    t = C.uniform_pairs(31, n, C.Q_NTT)
    y = C.uniform_pairs(32, 8 * n, C.Q_NTT)
    want = C.oracle_ntt_inverse(y, t, logn)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    assert np.array_equal(inverse(ctx, p, y, inplace=True), want)
    pu = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t[:, ::-1].copy(), bn.LAYOUT_U128)
    assert np.array_equal(inverse(ctx, pu, y[:, ::-1].copy())[:, ::-1], want)
    p.close()
    pu.close()


@pytest.mark.parametrize("logn", [3, 8, 10, 13, 17])
def test_negacyclic_polynomial_product(ctx, logn):
    """a * b mod (x^N + 1) by forward transforms, the fused pointwise product
    and the inverse, against schoolbook (N <= 2^10) or the oracle."""
    n = 1 << logn
    psi = pow(ROOT21, 1 << (C.NC_LOG2_ORDER - logn - 1), Q_NC)
    p = bn.Plan.negacyclic(ctx, logn, Q_NC, MU_NC, psi)
    a = C.uniform_pairs(41, n, Q_NC)
    b = C.uniform_pairs(42, n, Q_NC)
    da, db = DevBuf.from_array(ctx, a), DevBuf.from_array(ctx, b)
    dbh, dc = DevBuf(ctx, a.nbytes), DevBuf(ctx, a.nbytes)
    L = bn.lib()
    bn.check(L.bntt_ntt_forward_dev(p.handle, dbh.ptr, db.ptr, 1))
    bn.check(L.bntt_ntt_forward_mul_dev(p.handle, dc.ptr, da.ptr, dbh.ptr, 1, 1))
    bn.check(L.bntt_ntt_inverse_dev(p.handle, dc.ptr, dc.ptr, 1))
    got = dc.to_array()
    if logn <= 10:
        want = C.to_pairs(C.negacyclic_mul(C.from_pairs(a), C.from_pairs(b), Q_NC))
    else:
        t = C.negacyclic_table(Q_NC, logn, psi)
        prod_hat = C.oracle_blas("vvmul", C.oracle_ntt(a, t, logn, Q_NC, MU_NC, form=1, threads=8),
                                 C.oracle_ntt(b, t, logn, Q_NC, MU_NC, form=1, threads=8), Q_NC, MU_NC)
        want = C.oracle_ntt_inverse(prod_hat, t, logn, Q_NC, MU_NC)
    assert np.array_equal(got, want)
    for d in (da, db, dbh, dc):
        d.free()
    p.close()


def test_inverse_argument_errors(ctx):
    L = bn.lib()
    q = (1 << 123) + 12345678901                      # not pseudo-Mersenne: no fast multiply
    p = bn.Plan(ctx, 4, q, (1 << 251) // q, C.uniform_pairs(1, 16, q))
    d = DevBuf(ctx, 16 * 16)
    assert L.bntt_ntt_inverse_dev(p.handle, d.ptr, d.ptr, 1) == bn.EINVAL
    p.close()
    t = C.uniform_pairs(2, 16, C.Q_NTT)
    t[5] = C.to_pairs([0])[0]                          # a twiddle with no inverse
    p = bn.Plan(ctx, 4, C.Q_NTT, C.MU_NTT, t)
    assert L.bntt_ntt_inverse_dev(p.handle, d.ptr, d.ptr, 1) == bn.EINVAL
    assert b"no inverse" in L.bntt_last_error()
    assert L.bntt_ntt_inverse_dev(p.handle, d.addr + 8, d.ptr, 1) == bn.EINVAL
    assert L.bntt_ntt_inverse_dev(p.handle, d.ptr, d.ptr, 0) == bn.OK
    d.free()
    p.close()


@pytest.mark.parametrize("logn", [21, 22, 24])
def test_round_trip_largest_sizes(ctx, logn):
    """Up to the largest plan (2^24 points, three HBM passes of 8 stages each
    way): ntt^-1(ntt(x)) = x for a random table, and the forward output is a
    different vector."""
    n = 1 << logn
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    x = C.uniform_pairs(9100 + logn, n, C.Q_NTT)
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, t)
    y = forward(ctx, p, x)
    assert not np.array_equal(y, x)
    assert np.array_equal(inverse(ctx, p, y), x)
    p.close()


def test_negacyclic_smallest_plan(ctx):
    """N = 2: psi of order 4, one butterfly, against the oracle and back."""
    psi = pow(ROOT21, 1 << (C.NC_LOG2_ORDER - 2), Q_NC)
    p = bn.Plan.negacyclic(ctx, 1, Q_NC, MU_NC, psi)
    x = C.uniform_pairs(5, 2 * 64, Q_NC)
    t = C.negacyclic_table(Q_NC, 1, psi)
    y = forward(ctx, p, x)
    assert np.array_equal(y, C.oracle_ntt(x, t, 1, Q_NC, MU_NC))
    assert np.array_equal(inverse(ctx, p, y), x)
    p.close()

"""GPU parity of the fused transform + pointwise product
(bntt_ntt_forward_mul_dev): y = vector_mul(ntt(x), b), i.e. the reference's
ntt() (src/ntt_scalar.c:582) followed by vector_mul() (src/blas_scalar.c:594)
under the plan's modulus.  Compared bit for bit (integer results) with the
oracle running the two steps one after the other.
"""
import ctypes

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from gpu_util import DevBuf

pytestmark = pytest.mark.gpu
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")
Q_NC = C.from_pairs(GEN["nc_q"])[0]
MU_NC = (1 << 251) // Q_NC
ROOT21 = C.from_pairs(GEN["nc_root21"])[0]


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


def fused(ctx, logn, t, x, b, per_transform, q=C.Q_NTT, mu=C.MU_NTT, layout=bn.LAYOUT_HILO,
          inplace=False):
    p = bn.Plan(ctx, logn, q, mu, t if layout == bn.LAYOUT_HILO else t[:, ::-1].copy(), layout)
    dx, db = DevBuf.from_array(ctx, x), DevBuf.from_array(ctx, b)
    dy = dx if inplace else DevBuf(ctx, x.nbytes)
    bn.check(bn.lib().bntt_ntt_forward_mul_dev(p.handle, dy.ptr, dx.ptr, db.ptr,
                                               1 if per_transform else 0,
                                               x.shape[0] >> logn))
    y = dy.to_array()
    for d in {id(dx): dx, id(db): db, id(dy): dy}.values():
        d.free()
    p.close()
    return y


def expected(logn, t, x, b, per_transform, q=C.Q_NTT, mu=C.MU_NTT):
    y = C.oracle_ntt(x, t, logn, q, mu, form=1, threads=8)
    if not per_transform:
        b = np.tile(b, (x.shape[0] >> logn, 1))
    return C.oracle_blas("vvmul", y, b, q, mu)


@pytest.mark.parametrize("logn,batch", [(1, 5), (4, 300), (7, 33), (10, 64), (11, 4), (13, 2),
                                        (16, 2), (20, 1)])
@pytest.mark.parametrize("per_transform", [True, False])
def test_fused_matches_ntt_then_vector_mul(ctx, logn, batch, per_transform):
    n = 1 << logn
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    x = C.uniform_pairs(1000 + logn, batch * n, C.Q_NTT)
    b = C.uniform_pairs(3000 + logn, (batch if per_transform else 1) * n, C.Q_NTT)
    got = fused(ctx, logn, t, x, b, per_transform)
    assert np.array_equal(got, expected(logn, t, x, b, per_transform))


@pytest.mark.parametrize("logn", [6, 12])
def test_fused_reference_arith_and_u128_layout(ctx, ctx_ref, logn):
    n = 1 << logn
    t = C.uniform_pairs(11, n, C.Q_NTT)
    x = C.uniform_pairs(12, 16 * n, C.Q_NTT)
    b = C.uniform_pairs(13, 16 * n, C.Q_NTT)
    want = expected(logn, t, x, b, True)
    assert np.array_equal(fused(ctx_ref, logn, t, x, b, True), want)
    u = fused(ctx, logn, t, x[:, ::-1].copy(), b[:, ::-1].copy(), True, layout=bn.LAYOUT_U128)
    assert np.array_equal(u[:, ::-1], want)


def test_fused_in_place(ctx):
    logn = 10
    t = C.uniform_pairs(21, 1 << logn, C.Q_NTT)
    x = C.uniform_pairs(22, 8 << logn, C.Q_NTT)
    b = C.uniform_pairs(23, 1 << logn, C.Q_NTT)
    assert np.array_equal(fused(ctx, logn, t, x, b, False, inplace=True),
                          expected(logn, t, x, b, False))


@pytest.mark.parametrize("logn", [5, 10, 14])
def test_polynomial_product_in_friendly_prime_mode(ctx, logn):
    """With root-power tables, ntt(a) o ntt(b) is the transform of the
    negacyclic product a * b mod (x^N + 1): the fused call gives it with one
    launch sequence (b pre-transformed)."""
    n = 1 << logn
    psi = pow(ROOT21, 1 << (C.NC_LOG2_ORDER - logn - 1), Q_NC)
    t = C.negacyclic_table(Q_NC, logn, psi)
    a = C.uniform_pairs(31, n, Q_NC)
    bb = C.uniform_pairs(32, n, Q_NC)
    b_hat = C.oracle_ntt(bb, t, logn, Q_NC, MU_NC)
    got = fused(ctx, logn, t, a, b_hat, True, Q_NC, MU_NC)
    if logn <= 10:
        prod = C.to_pairs(C.negacyclic_mul(C.from_pairs(a), C.from_pairs(bb), Q_NC))
        assert np.array_equal(got, C.oracle_ntt(prod, t, logn, Q_NC, MU_NC))
    assert np.array_equal(got, expected(logn, t, a, b_hat, True, Q_NC, MU_NC))


def test_fused_argument_errors(ctx):
    logn = 6
    p = bn.Plan(ctx, logn, C.Q_NTT, C.MU_NTT, C.uniform_pairs(1, 64, C.Q_NTT))
    d = DevBuf(ctx, 64 * 16 * 4)
    L = bn.lib()
    assert L.bntt_ntt_forward_mul_dev(p.handle, d.ptr, d.ptr, None, 1, 1) == bn.EINVAL
    # b overlapping y is refused
    assert L.bntt_ntt_forward_mul_dev(p.handle, d.ptr, d.ptr, d.addr + 16 * 32, 0, 1) == bn.EINVAL
    assert b"overlap" in L.bntt_last_error()
    assert L.bntt_ntt_forward_mul_dev(p.handle, d.ptr, d.ptr, d.addr + 16 * 64, 2, 1) == bn.EINVAL
    assert L.bntt_ntt_forward_mul_dev(p.handle, d.ptr, d.ptr, d.addr + 8, 0, 1) == bn.EINVAL
    assert L.bntt_ntt_forward_mul_dev(p.handle, d.ptr, d.ptr, d.addr + 16 * 64, 0, 0) == bn.OK
    d.free()
    p.close()

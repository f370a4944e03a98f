"""GPU parity of vvadd / vvsub / vvmul / axpy (src/blas_scalar.c:578-608).

Bit-exact comparisons (integer work: tolerance 0) against the reference's
golden vectors, fixtures produced by the compiled reference, and the oracle.
"""
import ctypes

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C
from gpu_util import DevBuf, dev_blas, hilo_to_u128, u128_to_hilo

pytestmark = pytest.mark.gpu

GOLD = C.load_golden()
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")
OPS = ["vvadd", "vvsub", "vvmul", "axpy"]


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


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("which", ["auto", "reference"])
def test_blas_reference_goldens_dev(ctx, ctx_ref, op, which):
    c = ctx if which == "auto" else ctx_ref
    a, b = GOLD["twd_1024"], GOLD["x_1024"]
    out = dev_blas(c, op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X)
    assert np.array_equal(out, GOLD[f"{op}_1024"])


@pytest.mark.parametrize("op", OPS)
def test_blas_reference_goldens_host(ctx, op):
    a, b = GOLD["twd_1024"], GOLD["x_1024"]
    out = np.empty_like(a)
    bn.blas(ctx, op, out, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X)
    assert np.array_equal(out, GOLD[f"{op}_1024"])


@pytest.mark.parametrize("op", OPS)
def test_blas_layout_u128(ctx, op):
    a, b = GOLD["twd_1024"], GOLD["x_1024"]
    out = dev_blas(ctx, op, hilo_to_u128(a), hilo_to_u128(b), C.Q_BLAS, C.MU_BLAS, C.AXPY_X,
                   layout=bn.LAYOUT_U128)
    assert np.array_equal(u128_to_hilo(out), GOLD[f"{op}_1024"])


@pytest.mark.parametrize("qname", ["ntt", "blas"])
@pytest.mark.parametrize("op", ["addmod", "submod", "mulmod"])
@pytest.mark.parametrize("which", ["auto", "reference"])
def test_arith_boundary_pairs_match_reference(ctx, ctx_ref, qname, op, which):
    """Boundary operands (0, 1, q-1, q, 2^64 +- 1, ...) of the reference's
    word arithmetic, including addmod's corner cases; outputs come from the
    compiled reference."""
    q, mu = (C.Q_NTT, C.MU_NTT) if qname == "ntt" else (C.Q_BLAS, C.MU_BLAS)
    a, b = GEN[f"arith_a_{qname}"], GEN[f"arith_b_{qname}"]
    blas_op = {"addmod": "vvadd", "submod": "vvsub", "mulmod": "vvmul"}[op]
    out = dev_blas(ctx if which == "auto" else ctx_ref, blas_op, a, b, q, mu)
    assert np.array_equal(out, GEN[f"arith_{op}_{qname}"])


def test_addmod_quirk_on_device(ctx):
    q = C.Q_NTT
    a = C.to_pairs([q - 1, 1, q])
    b = C.to_pairs([(1 << 64) + 1, q - 1, 1 << 64])
    out = C.from_pairs(dev_blas(ctx, "vvadd", a, b, q, C.MU_NTT))
    assert out == [0, q, 0]


@pytest.mark.parametrize("op", OPS)
def test_reference_arith_full_range_random(ctx_ref, op):
    """ARITH_REFERENCE replicates the reference for any 128-bit operands,
    including values outside [0, q)."""
    rng = np.random.default_rng(3)
    n = 1 << 14
    a = rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)
    b = rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)
    x = (1 << 127) + 12345
    out = dev_blas(ctx_ref, op, a, b, C.Q_BLAS, C.MU_BLAS, x)
    assert np.array_equal(out, C.oracle_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, x))


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("q", [(1 << 123) + 12345678901, (1 << 124) - 3, (1 << 124) - 0x7bfffff,
                               (1 << 124) - ((1 << 31) - 1), (1 << 100) + 7])
def test_other_moduli_match_oracle(ctx, op, q):
    mu = (1 << 251) // q if q > (1 << 123) else ((1 << 251) // q) & ((1 << 128) - 1)
    n = 5000
    a = C.uniform_pairs(31, n, q)
    b = C.uniform_pairs(32, n, q)
    x = C.from_pairs(C.uniform_pairs(33, 1, q))[0]
    out = dev_blas(ctx, op, a, b, q, mu, x)
    assert np.array_equal(out, C.oracle_blas(op, a, b, q, mu, x))


@pytest.mark.parametrize("n", [1, 3, 255, 1023, 1025, 4097])
def test_ragged_lengths(ctx, n):
    a = C.uniform_pairs(41, n, C.Q_BLAS)
    b = C.uniform_pairs(42, n, C.Q_BLAS)
    for op in OPS:
        out = dev_blas(ctx, op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X)
        assert np.array_equal(out, C.oracle_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X))


def test_zero_length_and_aliasing(ctx):
    m = bn.modulus(C.Q_BLAS, C.MU_BLAS)
    bn.check(bn.lib().bntt_vvmul_dev(ctx.handle, None, None, None, 0, ctypes.byref(m), 0))
    a = C.uniform_pairs(51, 3000, C.Q_BLAS)
    b = C.uniform_pairs(52, 3000, C.Q_BLAS)
    da, db = DevBuf.from_array(ctx, a), DevBuf.from_array(ctx, b)
    # c aliases a
    bn.check(bn.lib().bntt_vvmul_dev(ctx.handle, da.ptr, da.ptr, db.ptr, 3000, ctypes.byref(m), 0))
    assert np.array_equal(da.to_array(), C.oracle_blas("vvmul", a, b, C.Q_BLAS, C.MU_BLAS))
    da.free()
    db.free()


def test_invalid_arguments(ctx):
    m = bn.modulus(C.Q_BLAS, C.MU_BLAS)
    L = bn.lib()
    assert L.bntt_vvadd_dev(ctx.handle, None, None, None, 5, ctypes.byref(m), 0) == bn.EINVAL
    d = DevBuf(ctx, 4096)
    assert L.bntt_vvadd_dev(ctx.handle, d.addr + 8, d.ptr, d.ptr, 5, ctypes.byref(m), 0) == bn.EINVAL
    assert L.bntt_vvadd_dev(ctx.handle, d.ptr, d.ptr, d.ptr, 5, ctypes.byref(m), 7) == bn.EINVAL
    assert b"aligned" in L.bntt_last_error() or b"layout" in L.bntt_last_error()
    d.free()


@pytest.mark.parametrize("op", OPS)
def test_full_size_2_24_matches_oracle(ctx, op):
    """The bench configuration: 2^24 elements, uniform operands from a seed,
    generated on the device; compared element for element with the oracle."""
    n = 1 << 24
    m = bn.modulus(C.Q_BLAS, C.MU_BLAS)
    L = bn.lib()
    da, db, dc = DevBuf(ctx, n * 16), DevBuf(ctx, n * 16), DevBuf(ctx, n * 16)
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, da.ptr, n, 3000, 0, ctypes.byref(m), 0))
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, db.ptr, n, 4000, 0, ctypes.byref(m), 0))
    fn = getattr(L, f"bntt_{op}_dev")
    if op == "axpy":
        bn.check(fn(ctx.handle, dc.ptr, da.ptr, db.ptr, bn.U128.of(C.AXPY_X), n, ctypes.byref(m), 0))
    else:
        bn.check(fn(ctx.handle, dc.ptr, da.ptr, db.ptr, n, ctypes.byref(m), 0))
    a, b, c = da.to_array(), db.to_array(), dc.to_array()
    # device generator == host generator
    assert np.array_equal(a[:4096], C.uniform_pairs(3000, 4096, C.Q_BLAS))
    assert np.array_equal(b[-4096:], C.uniform_pairs(4000, 4096, C.Q_BLAS, offset=n - 4096))
    assert np.array_equal(c, C.oracle_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X))
    for d in (da, db, dc):
        d.free()

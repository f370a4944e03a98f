"""Pins the oracle (oracle/bntt_oracle.c) to the reference.

1. The reference's own golden vectors (data/ver_N.txt, data/<op>_1024.txt).
2. Fixtures the reference's compiled functions produced (tests/golden/ref_gen.npz).
3. When oracle/_ref is built, live differential fuzzing against the reference.
"""
import hashlib
import itertools
import random

import numpy as np
import pytest

import common as C

GOLD = C.load_golden()
GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.mark.parametrize("logn", range(4, 11))
@pytest.mark.parametrize("form", [0, 1])
def test_oracle_ntt_matches_reference_goldens(logn, form):
    n = 1 << logn
    y = C.oracle_ntt(GOLD[f"x_{n}"], GOLD[f"twd_{n}"], logn, form=form)
    assert np.array_equal(y, GOLD[f"ver_{n}"])


@pytest.mark.parametrize("op", ["vvadd", "vvsub", "vvmul", "axpy"])
def test_oracle_blas_matches_reference_goldens(op):
    # the BLAS driver uses a = twd_1024, b = x_1024 (src/blas_scalar.c:616-636)
    a, b = GOLD["twd_1024"], GOLD["x_1024"]
    c = C.oracle_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X)
    assert np.array_equal(c, GOLD[f"{op}_1024"])


@pytest.mark.parametrize("logn", range(2, 21))
def test_oracle_ntt_matches_reference_generated(logn):
    n = 1 << logn
    x = C.uniform_pairs(1000 + logn, n, C.Q_NTT)
    t = C.uniform_pairs(2000 + logn, n, C.Q_NTT)
    y = C.oracle_ntt(x, t, logn, form=1 if logn > 12 else 0)
    if logn <= 12:
        assert np.array_equal(y, GEN[f"ntt_y_{logn}"])
    assert sha(y) == str(GEN[f"ntt_sha_{logn}"])


@pytest.mark.parametrize("logn", [4, 7, 10])
@pytest.mark.parametrize("edge", ["zero", "one", "qm1", "q", "two64", "tqm1"])
def test_oracle_ntt_edge_inputs(logn, edge):
    n = 1 << logn
    q = C.Q_NTT
    x = C.uniform_pairs(1000 + logn, n, q)
    t = C.uniform_pairs(2000 + logn, n, q)
    vals = {"zero": 0, "one": 1, "qm1": q - 1, "q": q, "two64": 1 << 64}
    if edge == "tqm1":
        t = C.to_pairs([q - 1] * n)
    else:
        x = C.to_pairs([vals[edge]] * n)
    y = C.oracle_ntt(x, t, logn)
    assert np.array_equal(y, GEN[f"edge_{edge}_{logn}"])


@pytest.mark.parametrize("op", ["vvadd", "vvsub", "vvmul", "axpy"])
def test_oracle_blas_matches_reference_generated(op):
    a = C.uniform_pairs(3000, 1 << 16, C.Q_BLAS)
    b = C.uniform_pairs(4000, 1 << 16, C.Q_BLAS)
    c = C.oracle_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X)
    assert sha(c) == str(GEN[f"blas_{op}_sha"])


@pytest.mark.parametrize("qname", ["ntt", "blas"])
@pytest.mark.parametrize("op", ["addmod", "submod", "mulmod"])
def test_oracle_arith_boundary_pairs(qname, op):
    q, mu = (C.Q_NTT, C.MU_NTT) if qname == "ntt" else (C.Q_BLAS, C.MU_BLAS)
    a = C.from_pairs(GEN[f"arith_a_{qname}"])
    b = C.from_pairs(GEN[f"arith_b_{qname}"])
    want = C.from_pairs(GEN[f"arith_{op}_{qname}"])
    got = [C.oracle_scalar(op, x, y, q, mu) for x, y in zip(a, b)]
    assert got == want


def test_addmod_low_word_quirk_is_reproduced():
    """addmod(q-1, 2^64+1): a+b = q + 2^64 > q and lo64(a+b) == lo64(q); the
    reference returns 0 where exact arithmetic gives 2^64
    (src/ntt_scalar.c:68-76)."""
    q = C.Q_NTT
    got = C.oracle_scalar("addmod", q - 1, (1 << 64) + 1, q)
    assert got == 0
    idx = [i for i, (x, y) in enumerate(zip(C.from_pairs(GEN["arith_a_ntt"]),
                                             C.from_pairs(GEN["arith_b_ntt"])))
           if x == q and y == 1 << 64]
    assert idx and C.from_pairs(GEN["arith_addmod_ntt"])[idx[0]] == 0


def test_strict_addmod_returns_q():
    """a + b == q is returned unreduced (strict '>' test, src/ntt_scalar.c:74-76)."""
    q = C.Q_NTT
    assert C.oracle_scalar("addmod", 1, q - 1, q) == q


_Q_NC = (1 << 124) - (62 * (1 << 21) - 1)      # NTT-friendly prime, 2^21 | q - 1
_Q_K31 = (1 << 124) - ((1 << 31) - 1)           # largest k the fast path accepts


@pytest.mark.parametrize("q,mu", [(C.Q_NTT, C.MU_NTT), (C.Q_BLAS, C.MU_BLAS),
                                  (_Q_NC, (1 << 251) // _Q_NC), (_Q_K31, (1 << 251) // _Q_K31)])
def test_reference_barrett_is_exact_on_domain(q, mu):
    """For q = 2^124 - k and mu = floor(2^251/q) the reference quotient is
    within one of the true quotient, so mulmod128 returns a*b mod q exactly for
    a, b in [0, q].  The GPU fast path relies on this."""
    assert mu == (1 << 251) // q
    rng = random.Random(7)
    vals = C.edge_values(q) + [rng.randrange(q) for _ in range(300)]
    for a, b in itertools.islice(itertools.product(vals, vals), 40000):
        assert C.oracle_scalar("mulmod", a, b, q, mu) == (a * b) % q


needs_ref = pytest.mark.skipif(not C.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("op", ["addmod", "submod", "mulmod"])
def test_oracle_fuzz_vs_reference_full_range(op):
    """Random 128-bit operands, in and out of [0, q): the restatement follows
    every truncation of the reference word arithmetic."""
    rng = np.random.default_rng(11)
    n = 20000
    a = rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)
    b = rng.integers(0, 2**64, size=(n, 2), dtype=np.uint64)
    # half of the cases in-range for the NTT modulus
    a[: n // 2, 0] &= np.uint64((1 << 60) - 1)
    b[: n // 2, 0] &= np.uint64((1 << 60) - 1)
    q, mu = C.Q_NTT, C.MU_NTT
    lib = C.ref_lib("ntt", "scalar", 10)
    out = np.zeros_like(a)
    lib.bntt_ref_arith_many({"addmod": 0, "submod": 1, "mulmod": 2}[op], out.ctypes.data,
                            a.ctypes.data, b.ctypes.data, n, C.hi(q), C.lo(q), C.hi(mu), C.lo(mu))
    A, B = C.from_pairs(a), C.from_pairs(b)
    for i in range(0, n, 7):
        assert C.oracle_scalar(op, A[i], B[i], q, mu) == C.from_pairs(out[i:i + 1])[0]


@needs_ref
@pytest.mark.parametrize("logn", [2, 3, 5, 9, 11, 14])
def test_oracle_ntt_vs_reference_random_moduli(logn):
    """Runtime modulus/mu are arguments of the reference ntt(); check another
    pseudo-Mersenne prime and a non-special modulus."""
    n = 1 << logn
    for q in ((1 << 124) - 3, (1 << 123) + 12345678901):
        mu = (1 << 251) // q
        x = C.uniform_pairs(77 + logn, n, q)
        t = C.uniform_pairs(88 + logn, n, q)
        assert np.array_equal(C.oracle_ntt(x, t, logn, q, mu), C.ref_ntt(x, t, logn, q, mu))


@needs_ref
@pytest.mark.parametrize("impl", ["avx2", "avx512"])
@pytest.mark.parametrize("logn", [4, 8, 10])
def test_simd_reference_builds_agree_on_random_inputs(impl, logn):
    """The SIMD builds are the timed CPU baseline; on uniform inputs they agree
    with the scalar path (their corner-case differences need contrived values)."""
    import os
    if impl == "avx512" and "avx512dq" not in open("/proc/cpuinfo").read():
        pytest.skip("host lacks AVX-512")
    n = 1 << logn
    x = C.uniform_pairs(5 + logn, 8 * n, C.Q_NTT)
    t = C.uniform_pairs(6 + logn, n, C.Q_NTT)
    assert np.array_equal(C.ref_ntt(x, t, logn, impl=impl, threads=2),
                          C.ref_ntt(x, t, logn, impl="scalar"))


@pytest.mark.parametrize("logn", range(4, 11))
def test_oracle_inverse_inverts_reference_goldens(logn):
    """The inverse restatement (no reference counterpart) maps the reference's
    golden outputs data/ver_N.txt back to its inputs data/x_N.txt."""
    n = 1 << logn
    assert np.array_equal(C.oracle_ntt_inverse(GOLD[f"ver_{n}"], GOLD[f"twd_{n}"], logn),
                          GOLD[f"x_{n}"])


@pytest.mark.parametrize("logn", [1, 2, 5, 12, 14])
def test_oracle_inverse_round_trip(logn):
    n = 1 << logn
    x = C.uniform_pairs(300 + logn, 3 * n, C.Q_NTT)
    t = C.uniform_pairs(400 + logn, n, C.Q_NTT)
    assert np.array_equal(C.oracle_ntt_inverse(C.oracle_ntt(x, t, logn, form=1), t, logn), x)

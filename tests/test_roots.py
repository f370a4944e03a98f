"""NTT-friendly prime mode on the host: prime search, roots of unity,
root-power tables, and the oracle's proof that the reference network with
such a table is the negacyclic NTT.

The reference ntt() (src/ntt_scalar.c:582) takes modulus, mu and table at
run time; tests/golden/ref_gen.npz holds its outputs (nc_*) for the prime
q = 2^124 - (62*2^21 - 1) and tables T[k] = psi^brv(k) built in pure Python.
Everything here is integer work: comparisons are exact.
"""
import ctypes
import hashlib
import random

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C

GEN = np.load(f"{C.GOLDEN}/ref_gen.npz")
Q_NC = C.from_pairs(GEN["nc_q"])[0]
MU_NC = (1 << 251) // Q_NC


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.mark.parametrize("t", [1, 10, 16, 21, 22, 24, 28])
def test_prime_search_matches_python(t):
    q, mu = bn.ntt_prime(t)
    assert q == C.ntt_prime_py(t)
    assert mu == (1 << 251) // q
    assert (q - 1) % (1 << t) == 0 and (1 << 124) - q < 1 << 28
    assert bn.lib().bntt_modulus_is_fast(ctypes.byref(bn.modulus(q, mu))) == 1


def test_fixture_prime_is_the_searched_one():
    assert Q_NC == bn.ntt_prime(C.NC_LOG2_ORDER)[0] == (1 << 124) - (62 * (1 << 21) - 1)
    # every smaller candidate has a Miller-Rabin witness (composite)
    for c in range(1, 62):
        assert not C.is_probable_prime((1 << 124) - (c * (1 << 21) - 1))


def test_smallest_order_one_prime_is_the_blas_modulus():
    """2^124 - 59 (src/blas_scalar.c:27) is the first prime below 2^124 of
    the form 2^124 - (2c - 1)."""
    assert bn.ntt_prime(1)[0] == C.Q_BLAS


def test_no_prime_in_range():
    with pytest.raises(bn.BnttError) as e:
        bn.ntt_prime(30)
    assert e.value.status == bn.EINVAL


@pytest.mark.parametrize("t", [1, 2, 11, 21])
def test_root_of_unity_has_exact_order(t):
    w = bn.root_of_unity(Q_NC, MU_NC, t)
    assert w == C.root_of_unity_py(Q_NC, t)
    assert pow(w, 1 << t, Q_NC) == 1
    assert pow(w, 1 << (t - 1), Q_NC) == Q_NC - 1
    assert C.from_pairs(GEN["nc_root21"])[0] == bn.root_of_unity(Q_NC, MU_NC, 21)


def test_root_of_unity_rejects_missing_order():
    # q_ntt - 1 = 2^124 - 720 = 2^4 * odd: roots of order up to 16 only
    assert bn.root_of_unity(C.Q_NTT, C.MU_NTT, 1) == C.Q_NTT - 1
    w = bn.root_of_unity(C.Q_NTT, C.MU_NTT, 4)
    assert pow(w, 8, C.Q_NTT) == C.Q_NTT - 1
    with pytest.raises(bn.BnttError):
        bn.root_of_unity(C.Q_NTT, C.MU_NTT, 5)
    with pytest.raises(bn.BnttError):
        bn.root_of_unity(Q_NC, MU_NC, 23)       # q - 1 = 2^22 * odd
    with pytest.raises(bn.BnttError):
        bn.root_of_unity(Q_NC, MU_NC + 1, 4)    # mu must be floor(2^251 / q)


def test_powmod_matches_python():
    rng = random.Random(5)
    for q in (Q_NC, C.Q_NTT, C.Q_BLAS, (1 << 123) + 12345678901):
        mu = (1 << 251) // q
        for _ in range(50):
            a, e = rng.randrange(q), rng.randrange(1 << 128)
            assert bn.powmod(q, mu, a, e) == pow(a, e, q)


@pytest.mark.parametrize("logn", [1, 2, 5, 10, 12])
@pytest.mark.parametrize("layout", [bn.LAYOUT_HILO, bn.LAYOUT_U128])
def test_host_table_matches_python(logn, layout):
    psi = C.negacyclic_psi(Q_NC, logn)
    t = bn.twiddles_negacyclic(Q_NC, MU_NC, logn, psi, layout)
    want = C.negacyclic_table(Q_NC, logn, psi)
    if layout == bn.LAYOUT_U128:
        want = want[:, ::-1]
    assert np.array_equal(t, want)


def test_table_rejects_non_primitive_psi():
    psi = C.negacyclic_psi(Q_NC, 6)
    with pytest.raises(bn.BnttError):
        bn.twiddles_negacyclic(Q_NC, MU_NC, 6, psi * psi % Q_NC)   # order N, not 2N
    with pytest.raises(bn.BnttError):
        bn.twiddles_negacyclic(Q_NC, MU_NC, 7, psi)                # order 2N for N = 64


@pytest.mark.parametrize("logn", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("form", [0, 1])
def test_reference_network_is_negacyclic_dft(logn, form):
    """Both network forms of the oracle (constant geometry, in place) with a
    root-power table compute Y[i] = sum_j X[j] psi^((2 brv(i) + 1) j)."""
    n = 1 << logn
    psi = C.negacyclic_psi(Q_NC, logn)
    x = C.uniform_pairs(77 + logn, n, Q_NC)
    y = C.oracle_ntt(x, C.negacyclic_table(Q_NC, logn, psi), logn, Q_NC, MU_NC, form=form)
    assert C.from_pairs(y) == C.negacyclic_dft(C.from_pairs(x), Q_NC, psi)


@pytest.mark.parametrize("logn", [3, 6, 8])
def test_convolution_theorem(logn):
    """NTT(a) o NTT(b) = NTT(a * b mod (x^N + 1)): the transform diagonalises
    negacyclic convolution."""
    n = 1 << logn
    psi = C.negacyclic_psi(Q_NC, logn)
    t = C.negacyclic_table(Q_NC, logn, psi)
    a = C.uniform_pairs(90, n, Q_NC)
    b = C.uniform_pairs(91, n, Q_NC)
    prod = C.to_pairs(C.negacyclic_mul(C.from_pairs(a), C.from_pairs(b), Q_NC))
    lhs = C.oracle_blas("vvmul", C.oracle_ntt(a, t, logn, Q_NC, MU_NC),
                        C.oracle_ntt(b, t, logn, Q_NC, MU_NC), Q_NC, MU_NC)
    assert np.array_equal(lhs, C.oracle_ntt(prod, t, logn, Q_NC, MU_NC))


@pytest.mark.parametrize("logn", range(2, 17))
def test_oracle_matches_reference_fixtures(logn):
    """The oracle reproduces the compiled reference's negacyclic outputs."""
    n = 1 << logn
    x = C.uniform_pairs(1000 + logn, n, Q_NC)
    t = C.negacyclic_table(Q_NC, logn, C.negacyclic_psi(Q_NC, logn))
    y = C.oracle_ntt(x, t, logn, Q_NC, MU_NC, form=1, threads=4)
    if logn <= 12:
        assert np.array_equal(y, GEN[f"nc_y_{logn}"])
    assert sha(y) == str(GEN[f"nc_sha_{logn}"])


@pytest.mark.skipif(not C.ref_available(), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("logn", [4, 9, 12])
def test_reference_live_with_friendly_prime(logn):
    """The reference ntt() compiled in place, run now with the friendly prime,
    equals the oracle on fresh random inputs."""
    n = 1 << logn
    t = C.negacyclic_table(Q_NC, logn, C.negacyclic_psi(Q_NC, logn))
    x = C.uniform_pairs(4242 + logn, 8 * n, Q_NC)
    assert np.array_equal(C.ref_ntt(x, t, logn, Q_NC, MU_NC),
                          C.oracle_ntt(x, t, logn, Q_NC, MU_NC, form=1))


def test_fast_multiply_bound_widened():
    """The pseudo-Mersenne path covers k < 2^28 (both reference moduli and
    every prime of this mode); k = 2^28 and a wrong mu fall back."""
    for k, fast in ((719, 1), (59, 1), ((1 << 28) - 1, 1), (1 << 28, 0), ((1 << 31) - 1, 0)):
        q = (1 << 124) - k
        assert bn.lib().bntt_modulus_is_fast(ctypes.byref(bn.modulus(q))) == fast
    q = (1 << 124) - 0x7bfffff
    assert bn.lib().bntt_modulus_is_fast(ctypes.byref(bn.modulus(q, ((1 << 251) // q) - 1))) == 0


@pytest.mark.parametrize("logn", [1, 3, 6])
def test_oracle_inverse_is_inverse_negacyclic_dft(logn):
    """With root-power tables the inverse network is
    x[j] = N^-1 sum_i Y[i] psi^-((2 brv(i) + 1) j)."""
    n = 1 << logn
    psi = C.negacyclic_psi(Q_NC, logn)
    y = C.uniform_pairs(61 + logn, n, Q_NC)
    got = C.from_pairs(C.oracle_ntt_inverse(y, C.negacyclic_table(Q_NC, logn, psi), logn,
                                            Q_NC, MU_NC))
    ys, ninv, pinv = C.from_pairs(y), pow(n, Q_NC - 2, Q_NC), pow(psi, Q_NC - 2, Q_NC)
    want = [ninv * sum(yi * pow(pinv, (2 * C.brv(i, logn) + 1) * j, Q_NC)
                       for i, yi in enumerate(ys)) % Q_NC for j in range(n)]
    assert got == want


@pytest.mark.parametrize("logn", [4, 8])
def test_oracle_polynomial_product(logn):
    n = 1 << logn
    t = C.negacyclic_table(Q_NC, logn, C.negacyclic_psi(Q_NC, logn))
    a, b = C.uniform_pairs(71, n, Q_NC), C.uniform_pairs(72, n, Q_NC)
    prod_hat = C.oracle_blas("vvmul", C.oracle_ntt(a, t, logn, Q_NC, MU_NC),
                             C.oracle_ntt(b, t, logn, Q_NC, MU_NC), Q_NC, MU_NC)
    got = C.oracle_ntt_inverse(prod_hat, t, logn, Q_NC, MU_NC)
    assert C.from_pairs(got) == C.negacyclic_mul(C.from_pairs(a), C.from_pairs(b), Q_NC)

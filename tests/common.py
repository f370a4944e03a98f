"""Shared helpers for the parity tests: reference constants, the seeded input
generator, hi-first pair conversions and loaders for the oracle libraries.

Values cross every boundary as "hi-first u64 pairs": an (n, 2) uint64 array
whose row i is (high 64 bits, low 64 bits) of element i, the layout of the
benchNTT data files (src/config.c:29-30).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

# NTT modulus / Barrett constant hard-coded in every NTT driver
# (src/ntt_scalar.c:632-633): q = 2^124 - 719, mu = floor(2^251 / q).
Q_NTT = (1152921504606846975 << 64) | 18446744073709550897
MU_NTT = (9223372036854775808 << 64) | 5752
# BLAS modulus (src/blas_scalar.c:23-30): q = 2^124 - 59, mu = 2^127 + 472.
Q_BLAS = (0x0FFFFFFFFFFFFFFF << 64) | 0xFFFFFFFFFFFFFFC5
MU_BLAS = (0x8000000000000000 << 64) | 0x1D8
# axpy scalar of the BLAS driver (src/blas_scalar.c:614).
AXPY_X = (208488538572646751 << 64) | 12808410693871070164

M64 = (1 << 64) - 1


def hi(v: int) -> int:
    return (v >> 64) & M64


def lo(v: int) -> int:
    return v & M64


def to_pairs(values) -> np.ndarray:
    """Python ints -> (n, 2) uint64 hi-first pairs."""
    out = np.empty((len(values), 2), dtype=np.uint64)
    for i, v in enumerate(values):
        out[i, 0] = hi(v)
        out[i, 1] = lo(v)
    return out


def from_pairs(arr: np.ndarray) -> list[int]:
    a = np.asarray(arr, dtype=np.uint64).reshape(-1, 2)
    return [(int(h) << 64) | int(l) for h, l in a]


# ----------------------------------------------------------------- generator
_GOLD = np.uint64(0x9E3779B97F4A7C15)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_pairs(seed: int, n: int, q: int, offset: int = 0) -> np.ndarray:
    """n values uniform in [0, q) as hi-first pairs, counter-based.

    Element i uses SplitMix64 outputs at counters 2(i+offset) (high word) and
    2(i+offset)+1 (low word); the 128-bit word is masked to bitlen(q) bits and
    q is subtracted once if it is still >= q.  The library's host and device
    generators produce the same values (bntt_fill_uniform)."""
    idx = np.arange(offset, offset + n, dtype=np.uint64)
    s = np.uint64(seed & M64)
    with np.errstate(over="ignore"):
        h = _mix(s + (np.uint64(2) * idx + np.uint64(1)) * _GOLD)
        l = _mix(s + (np.uint64(2) * idx + np.uint64(2)) * _GOLD)
    L = q.bit_length()
    if L <= 64:
        h[:] = 0
        if L < 64:
            l &= np.uint64((1 << L) - 1)
    elif L < 128:
        h &= np.uint64((1 << (L - 64)) - 1)
    out = np.stack([h, l], axis=1)
    # subtract q where value >= q (vectorised 128-bit compare/subtract)
    qh, ql = np.uint64(hi(q)), np.uint64(lo(q))
    ge = (out[:, 0] > qh) | ((out[:, 0] == qh) & (out[:, 1] >= ql))
    if ge.any():
        nl = out[ge, 1] - ql
        borrow = (out[ge, 1] < ql).astype(np.uint64)
        out[ge, 0] = out[ge, 0] - qh - borrow
        out[ge, 1] = nl
    return out


# ------------------------------------------------------------------- loaders
def load_golden():
    return np.load(os.path.join(GOLDEN, "ref_data.npz"))


_ORACLE = None


def oracle():
    """ctypes handle to oracle/liboracle.so (built by `make -C oracle`)."""
    global _ORACLE
    if _ORACLE is None:
        path = os.path.join(ORACLE_DIR, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        lib = ctypes.CDLL(path)
        u64 = ctypes.c_uint64
        p = ctypes.c_void_p
        for name in ("orc_addmod_pairs", "orc_submod_pairs", "orc_mulmod_pairs",
                     "orc_mulmod_exact_pairs"):
            getattr(lib, name).argtypes = [p] + [u64] * 8
            getattr(lib, name).restype = None
        lib.orc_ntt_batch.argtypes = [p, p, p, ctypes.c_int, ctypes.c_size_t,
                                      u64, u64, u64, u64, ctypes.c_int, ctypes.c_int]
        lib.orc_ntt_jobs.argtypes = [p, p, p, p, ctypes.c_size_t,
                                     u64, u64, u64, u64, ctypes.c_int, ctypes.c_int]
        lib.orc_ntt_inverse_batch.argtypes = [p, p, p, ctypes.c_int, ctypes.c_size_t,
                                              u64, u64, u64, u64]
        lib.orc_ntt_inverse_batch.restype = ctypes.c_int
        lib.orc_vvadd.argtypes = [p, p, p, ctypes.c_size_t, u64, u64]
        lib.orc_vvsub.argtypes = [p, p, p, ctypes.c_size_t, u64, u64]
        lib.orc_vvmul.argtypes = [p, p, p, ctypes.c_size_t, u64, u64, u64, u64]
        lib.orc_axpy.argtypes = [p, p, p, u64, u64, ctypes.c_size_t, u64, u64, u64, u64]
        _ORACLE = lib
    return _ORACLE


def _ptr(a: np.ndarray) -> int:
    assert a.flags.c_contiguous and a.dtype == np.uint64
    return a.ctypes.data


def oracle_scalar(op: str, a: int, b: int, q: int, mu: int = 0) -> int:
    lib = oracle()
    out = np.zeros(2, dtype=np.uint64)
    fn = getattr(lib, f"orc_{op}_pairs")
    fn(_ptr(out), hi(a), lo(a), hi(b), lo(b), hi(q), lo(q), hi(mu), lo(mu))
    return (int(out[0]) << 64) | int(out[1])


def oracle_ntt(x: np.ndarray, t: np.ndarray, logn: int, q: int = Q_NTT, mu: int = MU_NTT,
               form: int = 0, threads: int = 1) -> np.ndarray:
    """Forward transform(s) of x (shape (batch*N, 2) or (N, 2)) sharing t."""
    lib = oracle()
    n = 1 << logn
    x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, 2)
    t = np.ascontiguousarray(t, dtype=np.uint64).reshape(-1, 2)
    assert x.shape[0] % n == 0 and t.shape[0] == n
    y = np.empty_like(x)
    lib.orc_ntt_batch(_ptr(y), _ptr(x), _ptr(t), logn, x.shape[0] // n,
                      hi(q), lo(q), hi(mu), lo(mu), form, threads)
    return y


def oracle_ntt_inverse(y: np.ndarray, t: np.ndarray, logn: int, q: int = Q_NTT,
                       mu: int = MU_NTT) -> np.ndarray:
    """Inverse of the in-place network for forward table t (the oracle's
    restatement of bntt_ntt_inverse_dev); y holds batch*N elements."""
    lib = oracle()
    n = 1 << logn
    y = np.ascontiguousarray(y, dtype=np.uint64).reshape(-1, 2)
    t = np.ascontiguousarray(t, dtype=np.uint64).reshape(-1, 2)
    assert y.shape[0] % n == 0 and t.shape[0] == n
    x = np.empty_like(y)
    rc = lib.orc_ntt_inverse_batch(_ptr(x), _ptr(y), _ptr(t), logn, y.shape[0] // n,
                                   hi(q), lo(q), hi(mu), lo(mu))
    assert rc == 0, "table entry or N not invertible"
    return x


def oracle_ntt_jobs(xs, ts, logns, q: int = Q_NTT, mu: int = MU_NTT, threads: int = 1):
    """Mixed-size transforms: lists of per-job input / table arrays."""
    lib = oracle()
    count = len(xs)
    ys = [np.empty_like(np.ascontiguousarray(x, dtype=np.uint64)) for x in xs]
    xs = [np.ascontiguousarray(x, dtype=np.uint64) for x in xs]
    ts = [np.ascontiguousarray(t, dtype=np.uint64) for t in ts]
    P = ctypes.c_void_p * count
    lib.orc_ntt_jobs(P(*[_ptr(y) for y in ys]), P(*[_ptr(x) for x in xs]),
                     P(*[_ptr(t) for t in ts]), (ctypes.c_int * count)(*logns), count,
                     hi(q), lo(q), hi(mu), lo(mu), 0, threads)
    return ys


def oracle_blas(op: str, a: np.ndarray, b: np.ndarray, q: int, mu: int, x: int = 0):
    lib = oracle()
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 2)
    b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, 2)
    c = np.empty_like(a)
    n = a.shape[0]
    if op == "vvadd":
        lib.orc_vvadd(_ptr(c), _ptr(a), _ptr(b), n, hi(q), lo(q))
    elif op == "vvsub":
        lib.orc_vvsub(_ptr(c), _ptr(a), _ptr(b), n, hi(q), lo(q))
    elif op == "vvmul":
        lib.orc_vvmul(_ptr(c), _ptr(a), _ptr(b), n, hi(q), lo(q), hi(mu), lo(mu))
    elif op == "axpy":
        lib.orc_axpy(_ptr(c), _ptr(a), _ptr(b), hi(x), lo(x), n, hi(q), lo(q), hi(mu), lo(mu))
    else:
        raise ValueError(op)
    return c


# ------------------------------------------------- reference built in place
def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_ntt_scalar_10.so"))


_REF_CACHE: dict = {}


def ref_lib(kind: str, impl: str, stages: int | None = None):
    """ctypes handle to oracle/_ref/libref_<kind>_<impl>[_<stages>].so."""
    name = f"libref_{kind}_{impl}" + (f"_{stages}" if stages is not None else "") + ".so"
    if name in _REF_CACHE:
        return _REF_CACHE[name]
    lib = ctypes.CDLL(os.path.join(REF_DIR, name))
    u64, p, i32 = ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int
    if kind == "ntt":
        lib.bntt_ref_ntt_batch.argtypes = [p, p, p, ctypes.c_size_t, u64, u64, u64, u64, i32]
        lib.bntt_ref_ntt_batch.restype = ctypes.c_double
        if impl == "scalar":
            for nm in ("bntt_ref_addmod", "bntt_ref_submod"):
                getattr(lib, nm).argtypes = [p] + [u64] * 6
            lib.bntt_ref_mulmod.argtypes = [p] + [u64] * 8
            lib.bntt_ref_arith_many.argtypes = [i32, p, p, p, ctypes.c_size_t, u64, u64, u64, u64]
    else:
        lib.bntt_ref_blas.argtypes = [i32, p, p, p, u64, u64, ctypes.c_size_t,
                                      u64, u64, u64, u64, i32]
        lib.bntt_ref_blas.restype = ctypes.c_double
    _REF_CACHE[name] = lib
    return lib


def ref_ntt(x: np.ndarray, t: np.ndarray, logn: int, q: int = Q_NTT, mu: int = MU_NTT,
            impl: str = "scalar", threads: int = 1) -> np.ndarray:
    lib = ref_lib("ntt", impl, logn)
    n = 1 << logn
    x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, 2)
    t = np.ascontiguousarray(t, dtype=np.uint64).reshape(-1, 2)
    y = np.empty_like(x)
    lib.bntt_ref_ntt_batch(_ptr(y), _ptr(x), _ptr(t), x.shape[0] // n,
                           hi(q), lo(q), hi(mu), lo(mu), threads)
    return y


BLAS_OPS = {"vvadd": 0, "vvsub": 1, "vvmul": 2, "axpy": 3}


def ref_blas(op: str, a: np.ndarray, b: np.ndarray, q: int, mu: int, x: int = 0,
             impl: str = "scalar", threads: int = 1) -> np.ndarray:
    lib = ref_lib("blas", impl)
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 2)
    b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, 2)
    c = np.empty_like(a)
    t = lib.bntt_ref_blas(BLAS_OPS[op], _ptr(c), _ptr(a), _ptr(b), hi(x), lo(x), a.shape[0],
                          hi(q), lo(q), hi(mu), lo(mu), threads)
    assert t >= 0
    return c


def ref_scalar(op: str, a: int, b: int, q: int, mu: int = 0) -> int:
    lib = ref_lib("ntt", "scalar", 10)
    out = np.zeros(2, dtype=np.uint64)
    if op == "mulmod":
        lib.bntt_ref_mulmod(_ptr(out), hi(a), lo(a), hi(b), lo(b), hi(q), lo(q), hi(mu), lo(mu))
    else:
        getattr(lib, f"bntt_ref_{op}")(_ptr(out), hi(a), lo(a), hi(b), lo(b), hi(q), lo(q))
    return (int(out[0]) << 64) | int(out[1])


def edge_values(q: int) -> list[int]:
    """Operands at the boundaries that matter for the 64-bit word arithmetic."""
    vals = {0, 1, 2, q - 1, q - 2, q, (1 << 64) - 1, 1 << 64, (1 << 64) + 1,
            q - (1 << 64), q - (1 << 64) + 1, lo(q), lo(q) + 1, hi(q) << 64,
            (hi(q) << 64) - 1, q >> 1, (q >> 1) + 1, (1 << 123), (1 << 123) - 1}
    return sorted(v for v in vals if 0 <= v <= q)


# ------------------------------------------------- NTT-friendly prime mode
# Pure-Python restatement (independent of libbntt) used to pin
# bntt_ntt_prime / bntt_root_of_unity / bntt_twiddles_negacyclic and to
# build the negacyclic fixtures from the compiled reference ntt().
MR_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73,
            79, 83, 89)
NC_LOG2_ORDER = 21   # 2^21 | q - 1: negacyclic transforms up to N = 2^20


def is_probable_prime(n: int) -> bool:
    for p in MR_BASES:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in MR_BASES:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def ntt_prime_py(log2_order: int) -> int:
    """Smallest-c prime 2^124 - (c*2^log2_order - 1) with k < 2^28."""
    c = 1
    while True:
        k = (c << log2_order) - 1
        assert k < 1 << 28, "no prime in range"
        if is_probable_prime((1 << 124) - k):
            return (1 << 124) - k
        c += 1


def root_of_unity_py(q: int, log2_order: int) -> int:
    for g in range(2, 4096):
        w = pow(g, (q - 1) >> log2_order, q)
        if pow(w, 1 << (log2_order - 1), q) == q - 1:
            return w
    raise ValueError("no root found")


def brv(k: int, n: int) -> int:
    return int(format(k, f"0{n}b")[::-1], 2) if n else 0


def negacyclic_table(q: int, logn: int, psi: int) -> np.ndarray:
    """T[k] = psi^brv(k), T[0] = 1, as (N, 2) hi-first pairs."""
    n = 1 << logn
    pw = [1] * n
    for j in range(1, n):
        pw[j] = pw[j - 1] * psi % q
    return to_pairs([pw[brv(k, logn)] for k in range(n)])


def negacyclic_psi(q: int, logn: int, log2_order: int = NC_LOG2_ORDER) -> int:
    """Primitive 2N-th root: the order-2^log2_order root to the 2^(order-n-1)."""
    w = root_of_unity_py(q, log2_order)
    return pow(w, 1 << (log2_order - logn - 1), q)


def negacyclic_dft(x: list[int], q: int, psi: int) -> list[int]:
    """Y[i] = sum_j x[j] psi^((2 brv(i) + 1) j): the definition, O(N^2)."""
    n = len(x)
    logn = n.bit_length() - 1
    out = []
    for i in range(n):
        r = pow(psi, 2 * brv(i, logn) + 1, q)
        acc, p = 0, 1
        for xj in x:
            acc = (acc + xj * p) % q
            p = p * r % q
        out.append(acc)
    return out


def negacyclic_mul(a: list[int], b: list[int], q: int) -> list[int]:
    """a * b mod (x^N + 1, q), schoolbook."""
    n = len(a)
    c = [0] * n
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j, bj in enumerate(b):
            k = i + j
            if k < n:
                c[k] = (c[k] + ai * bj) % q
            else:
                c[k - n] = (c[k - n] - ai * bj) % q
    return c

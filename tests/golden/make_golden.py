"""Regenerates the committed parity fixtures in tests/golden/.

Run with BNTT_REF_ROOT naming the benchNTT source tree, after building the
reference in place (`make -C oracle ref REF_ROOT=$BNTT_REF_ROOT`):

    BNTT_REF_ROOT=<benchNTT> python tests/golden/make_golden.py

Writes:
  ref_data.npz   the reference's own golden vectors, converted from text:
                 x_N, twd_N, ver_N for N = 16..1024 (data/{x,twd,ver}_N.txt)
                 and vvadd/vvsub/vvmul/axpy_1024 (data/<op>_1024.txt), each an
                 (N, 2) uint64 array of hi-first pairs (src/config.c:17-31).
  ref_gen.npz    outputs of the reference functions themselves (compiled from
                 the sources by oracle/Makefile) on seeded inputs the tests can
                 regenerate with tests/common.uniform_pairs:
                   ntt_y_<logn>      full outputs, logn = 1..12 (scalar ntt(),
                                     src/ntt_scalar.c:582)
                   ntt_sha_<logn>    SHA-256 of the output bytes, logn = 13..20
                   edge_*            transforms of boundary inputs (all 0,
                                     all q-1, all q, ...)
                   blas_<op>_sha     SHA-256 of each BLAS op at 2^16 elements
                   arith_*           add/sub/mul of boundary operand pairs
                   nc_*              NTT-friendly prime mode: the reference
                                     ntt() run with q = 2^124 - (62*2^21 - 1),
                                     mu = floor(2^251/q) and root-power tables
                                     T[k] = psi^brv(k) (computed here in pure
                                     Python): nc_y_<logn> (2..12), nc_sha_<logn>
                                     (13..20), nc_q, nc_root21
"""
from __future__ import annotations

import hashlib
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import common as C  # noqa: E402

REF_ROOT = os.environ.get("BNTT_REF_ROOT", "")

# Seeds of the generated fixtures (tests regenerate the same inputs).
SEED_X = 1000
SEED_T = 2000
SEED_A = 3000
SEED_B = 4000
BLAS_LEN = 1 << 16


def read_pairs(path: str, n: int) -> np.ndarray:
    vals = np.loadtxt(path, dtype=np.uint64)
    assert vals.shape[0] >= 2 * n, path
    return vals[: 2 * n].reshape(n, 2)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def gen_inputs(logn: int, q: int = C.Q_NTT):
    n = 1 << logn
    return C.uniform_pairs(SEED_X + logn, n, q), C.uniform_pairs(SEED_T + logn, n, q)


def main() -> None:
    if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "data")):
        sys.exit("set BNTT_REF_ROOT to the benchNTT source tree (the directory holding data/ and src/)")
    data = os.path.join(REF_ROOT, "data")
    out = {}
    for logn in range(4, 11):
        n = 1 << logn
        for kind in ("x", "twd", "ver"):
            out[f"{kind}_{n}"] = read_pairs(os.path.join(data, f"{kind}_{n}.txt"), n)
    for op in ("vvadd", "vvsub", "vvmul", "axpy"):
        out[f"{op}_1024"] = read_pairs(os.path.join(data, f"{op}_1024.txt"), 1024)
    np.savez_compressed(os.path.join(HERE, "ref_data.npz"), **out)

    if not C.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    gen = {}
    for logn in range(2, 21):
        x, t = gen_inputs(logn)
        y = C.ref_ntt(x, t, logn, threads=8)
        if logn <= 12:
            gen[f"ntt_y_{logn}"] = y
        gen[f"ntt_sha_{logn}"] = np.array(sha(y))
    q = C.Q_NTT
    edges = {"zero": 0, "one": 1, "qm1": q - 1, "q": q, "two64": 1 << 64}
    for logn in (4, 7, 10):
        n = 1 << logn
        _, t = gen_inputs(logn)
        for name, v in edges.items():
            x = C.to_pairs([v] * n)
            gen[f"edge_{name}_{logn}"] = C.ref_ntt(x, t, logn)
        # table of all q-1 against random data
        x, _ = gen_inputs(logn)
        tq = C.to_pairs([q - 1] * n)
        gen[f"edge_tqm1_{logn}"] = C.ref_ntt(x, tq, logn)
    a = C.uniform_pairs(SEED_A, BLAS_LEN, C.Q_BLAS)
    b = C.uniform_pairs(SEED_B, BLAS_LEN, C.Q_BLAS)
    for op in ("vvadd", "vvsub", "vvmul", "axpy"):
        c = C.ref_blas(op, a, b, C.Q_BLAS, C.MU_BLAS, C.AXPY_X, threads=8)
        gen[f"blas_{op}_sha"] = np.array(sha(c))
    for qname, qq, mu in (("ntt", C.Q_NTT, C.MU_NTT), ("blas", C.Q_BLAS, C.MU_BLAS)):
        ev = C.edge_values(qq)
        pa = [p[0] for p in itertools.product(ev, ev)]
        pb = [p[1] for p in itertools.product(ev, ev)]
        gen[f"arith_a_{qname}"] = C.to_pairs(pa)
        gen[f"arith_b_{qname}"] = C.to_pairs(pb)
        for op in ("addmod", "submod", "mulmod"):
            gen[f"arith_{op}_{qname}"] = C.to_pairs(
                [C.ref_scalar(op, x, y, qq, mu) for x, y in zip(pa, pb)])
    qn = C.ntt_prime_py(C.NC_LOG2_ORDER)
    mun = (1 << 251) // qn
    gen["nc_q"] = C.to_pairs([qn])
    gen["nc_root21"] = C.to_pairs([C.root_of_unity_py(qn, C.NC_LOG2_ORDER)])
    for logn in range(2, 21):
        n = 1 << logn
        x = C.uniform_pairs(SEED_X + logn, n, qn)
        t = C.negacyclic_table(qn, logn, C.negacyclic_psi(qn, logn))
        y = C.ref_ntt(x, t, logn, qn, mun, threads=8)
        if logn <= 12:
            gen[f"nc_y_{logn}"] = y
        gen[f"nc_sha_{logn}"] = np.array(sha(y))
    np.savez_compressed(os.path.join(HERE, "ref_gen.npz"), **gen)
    print("wrote", sorted(out), "and", len(gen), "generated fixtures")


if __name__ == "__main__":
    main()

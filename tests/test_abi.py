"""CPU checks of the C ABI: the library builds, loads without a GPU, and
exports every function include/bntt.h declares.  No compute calls."""
import ctypes
import os
import re
import subprocess

import pytest

import benchntt_b200 as bn
import common as C

HEADER = os.path.join(C.ROOT, "include", "bntt.h")


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bntt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_api():
    names = declared_functions(HEADER)
    for must in ("bntt_ctx_create", "bntt_plan_create", "bntt_ntt_forward_dev",
                 "bntt_batch_run_dev", "bntt_vvmul_dev", "bntt_axpy_host"):
        assert must in names


def all_headers():
    inc = os.path.join(C.ROOT, "include")
    return [os.path.join(inc, f) for f in sorted(os.listdir(inc)) if f.endswith(".h")]


def test_library_exports_every_declared_symbol():
    lib = bn.lib()
    for h in all_headers():
        # trailing-underscore names are header-local helpers (static inline)
        names = [n for n in declared_functions(h) if not n.endswith("_")]
        missing = [n for n in names if not hasattr(lib, n)]
        assert not missing, (h, missing)


def test_compat_headers_compile_as_c():
    """The reference's C drivers compile against the compat headers."""
    for src, extra in (("ntt_scalar_driver.c", ["-Dstages=8"]),
                       ("ntt_simd_driver.c", ["-Dstages=8", "-mavx2"]),
                       ("ntt_avx512_driver.c", ["-Dstages=8", "-mavx512f", "-mavx512dq"]),
                       ("blas_driver.c", []),
                       ("blas_simd_driver.c", ["-mavx2"]),
                       ("blas_simd_driver.c", ["-mavx512f", "-mavx512dq", "-DBNTT_DRIVER_AVX512"])):
        subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", *extra, "-I",
                        os.path.join(C.ROOT, "include"),
                        os.path.join(C.ROOT, "tests", "compat", src)], check=True)


def test_only_bntt_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", bn.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    syms = [l.split()[-1] for l in out.splitlines() if l.split()[1] in ("T", "D", "B")]
    assert syms and all(s.startswith("bntt_") for s in syms), [s for s in syms if not s.startswith("bntt_")][:5]


def test_python_binding_covers_header():
    assert set(declared_functions(HEADER)) <= set(bn.exported_symbols())


def test_status_strings_and_reference_moduli():
    lib = bn.lib()
    assert lib.bntt_status_string(bn.EBUDGET) == b"HBM budget exceeded"
    m = lib.bntt_modulus_ntt_reference()
    assert (m.q.hi << 64 | m.q.lo) == C.Q_NTT and (m.mu.hi << 64 | m.mu.lo) == C.MU_NTT
    m = lib.bntt_modulus_blas_reference()
    assert (m.q.hi << 64 | m.q.lo) == C.Q_BLAS and (m.mu.hi << 64 | m.mu.lo) == C.MU_BLAS


@pytest.mark.parametrize("q,fast", [(C.Q_NTT, 1), (C.Q_BLAS, 1), ((1 << 124) - 3, 1),
                                    ((1 << 124) - (1 << 14), 1), ((1 << 124) - (1 << 28) + 1, 1),
                                    ((1 << 124) - (1 << 28), 0), ((1 << 124) - (1 << 31) + 1, 0), ((1 << 123) + 5, 0),
                                    ((1 << 127) + 99, 0)])
def test_fast_path_eligibility(q, fast):
    mu = ((1 << 251) // q) & ((1 << 128) - 1)
    m = bn.modulus(q, mu)
    assert bn.lib().bntt_modulus_is_fast(ctypes.byref(m)) == fast
    wrong = bn.modulus(q, mu ^ 1)
    assert bn.lib().bntt_modulus_is_fast(ctypes.byref(wrong)) == 0


def test_host_generator_matches_test_generator():
    for q in (C.Q_NTT, C.Q_BLAS, (1 << 127) + 99, 1000003, (1 << 64) + 13):
        assert (bn.fill_uniform(17, 999, q, offset=5) == C.uniform_pairs(17, 999, q, offset=5)).all()


def test_ctx_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    rc = bn.lib().bntt_ctx_create(ctypes.byref(h), 0, None)
    assert rc == bn.ENODEV and not h.value
    assert b"no CUDA device" in bn.lib().bntt_last_error()


def test_no_unordered_copies_in_library_sources():
    """Kernels run on each context's non-blocking stream.  A plain cudaMemcpy /
    cudaMemcpy2D / cudaMemset goes to the legacy default stream, which is not
    ordered with such a stream (and from pageable memory may return before the
    data lands), so library code uses the Async forms on the context's stream.
    The one plain copy allowed reads a status word after its stream was
    synchronized."""
    import glob
    import re
    allowed = {("batch.cu", "cudaMemcpy(&err")}
    pat = re.compile(r"\b(cudaMemcpy|cudaMemcpy2D|cudaMemset)\(")
    found = []
    for path in sorted(glob.glob(os.path.join(C.ROOT, "benchntt_b200", "csrc", "*.cu"))):
        for line in open(path):
            if pat.search(line) and not any(os.path.basename(path) == f and tok in line
                                            for f, tok in allowed):
                found.append(f"{os.path.basename(path)}: {line.strip()}")
    assert not found, found

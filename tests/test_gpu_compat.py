"""C programs in the shape of the reference drivers, linked against libbntt
through include/bntt_compat.h and include/bntt_compat_simd.h, on the
reference's golden data written in its text format."""
import os
import subprocess

import numpy as np
import pytest

import benchntt_b200 as bn
import common as C

pytestmark = pytest.mark.gpu
SRC = os.path.join(C.ROOT, "tests", "compat")
LIBDIR = os.path.dirname(bn.LIB_PATH)


@pytest.fixture(scope="module")
def datadir(tmp_path_factory):
    d = tmp_path_factory.mktemp("data")
    gold = C.load_golden()
    for key in gold.files:   # x_N, twd_N, ver_N, <op>_1024: one decimal u64 per line
        np.savetxt(d / f"{key}.txt", gold[key].reshape(-1), fmt="%d")
    return str(d)


def build(tmp_path, src, extra=()):
    exe = str(tmp_path / (os.path.basename(src) + "".join(extra).replace("-", "_") + ".bin"))
    subprocess.run(["gcc", "-O2", "-std=gnu11", *extra, "-I", os.path.join(C.ROOT, "include"),
                    os.path.join(SRC, src), "-L", LIBDIR, "-lbntt", f"-Wl,-rpath,{LIBDIR}",
                    "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("stages", [4, 7, 10])
def test_scalar_ntt_driver(tmp_path, datadir, stages):
    exe = build(tmp_path, "ntt_scalar_driver.c", (f"-Dstages={stages}",))
    out = subprocess.run([exe, datadir], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == f"{1 << stages} fail: 0"


@pytest.mark.parametrize("stages", [5, 10])
def test_simd_ntt_driver(tmp_path, datadir, stages):
    exe = build(tmp_path, "ntt_simd_driver.c", (f"-Dstages={stages}", "-mavx2"))
    out = subprocess.run([exe, datadir], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == f"{1 << stages} fail: 0"


def host_has(*flags) -> bool:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                have = set(line.split(":", 1)[1].split())
                return all(f in have for f in flags)
    except OSError:
        pass
    return False


AVX512 = ("-mavx512f", "-mavx512dq")
needs_avx512 = pytest.mark.skipif(not host_has("avx512f", "avx512dq"), reason="host CPU lacks AVX-512F/DQ")


@needs_avx512
@pytest.mark.parametrize("stages", [4, 7, 10])
def test_avx512_ntt_driver(tmp_path, datadir, stages):
    """The 8-lane driver's call shape: ntt_pre with the permutation vectors,
    the 16-argument ntt (src/ntt_avx512.c:461, driver :580-594)."""
    exe = build(tmp_path, "ntt_avx512_driver.c", (f"-Dstages={stages}", *AVX512))
    out = subprocess.run([exe, datadir], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == f"{1 << stages} fail: 0"


@pytest.mark.parametrize("isa", ["avx2", "avx512"])
def test_simd_blas_driver(tmp_path, datadir, isa):
    """vector_add(c, a, b, mh, ml) ... axpy(c, a, b, xh, xl, mh, ml, muh, mul)
    on __m256i / __m512i arrays (src/blas_avx2.c:448-523,
    src/blas_avx512.c:401-476)."""
    if isa == "avx512" and not host_has("avx512f", "avx512dq"):
        pytest.skip("host CPU lacks AVX-512F/DQ")
    if isa == "avx2" and not host_has("avx2"):
        pytest.skip("host CPU lacks AVX2")
    flags = (*AVX512, "-DBNTT_DRIVER_AVX512") if isa == "avx512" else ("-mavx2",)
    exe = build(tmp_path, "blas_simd_driver.c", flags)
    out = subprocess.run([exe, datadir], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split() == ["vvadd", "fail:", "0", "vvsub", "fail:", "0", "vvmul", "fail:",
                                  "0", "axpy", "fail:", "0"]


def test_blas_driver(tmp_path, datadir):
    exe = build(tmp_path, "blas_driver.c")
    out = subprocess.run([exe, datadir], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split() == ["vvadd", "fail:", "0", "vvsub", "fail:", "0", "vvmul", "fail:",
                                  "0", "axpy", "fail:", "0"]


@pytest.mark.parametrize("logn,batch", [(3, 3), (6, 2), (9, 1)])
def test_polymul_driver(tmp_path, logn, batch):
    """A C program on the native ABI: negacyclic products through forward,
    fused pointwise product and inverse, against its own schoolbook product."""
    exe = build(tmp_path, "polymul_driver.c")
    out = subprocess.run([exe, str(logn), str(batch)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == f"{1 << logn} fail: 0"


@pytest.mark.parametrize("runs,jobs", [(1, 10), (4, 40)])
def test_batch_host_driver(tmp_path, runs, jobs):
    """A C program on the native ABI: mixed-size host-buffer batches queued
    back to back (bntt_batch_run_host_async, one bntt_batch_sync), every job
    equal to the plan's single-transform host call."""
    exe = build(tmp_path, "batch_host_driver.c")
    out = subprocess.run([exe, str(runs), str(jobs)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "fail: 0"

"""The CPU baseline and bench.py's reference arm (no GPU needed).

They time the reference's own code built in place (oracle/_ref).  These
checks confirm that the job-list runner computes what the oracle computes, in
both timed forms, and that the reference arm prints the same workload config
as the GPU arm and never loads the product library.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import common as C
from benchntt_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_cpu as R  # noqa: E402

needs_ref = pytest.mark.skipif(R.best_impl() is None, reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("mode", ["ntt_only", "full"])
def test_job_runner_matches_oracle(mode):
    logns = [4, 10, 5, 16, 9, 4, 12, 7, 6, 8, 11, 4]
    rb = R.RefNttBatch(logns, C.Q_NTT, C.MU_NTT, W.SEED_TWIDDLE_BASE, 9, elems_per_task=64)
    rb.run(mode, 3)
    y = rb.y
    if mode == "ntt_only" and rb.impl == "scalar":   # native uint128_t output
        y = np.ascontiguousarray(y[:, ::-1])
    pos = 0
    for n in sorted(logns, reverse=True):
        x = np.ascontiguousarray(rb.x[pos:pos + (1 << n)])
        want = C.oracle_ntt(x, rb.tables[n], n, threads=2)
        assert np.array_equal(y[pos:pos + (1 << n)], want), f"2^{n} ({mode})"
        pos += 1 << n
    rb.close()


@needs_ref
def test_blas_runner_matches_oracle():
    blas = R.RefBlas("scalar")
    n = 4096
    a = R.uniform_pairs(1, n, C.Q_BLAS)
    b = R.uniform_pairs(2, n, C.Q_BLAS)
    c = R.aligned_pairs(n)
    for op in ("vvadd", "vvsub", "vvmul", "axpy"):
        blas.run(op, c, a, b, C.AXPY_X, C.Q_BLAS, C.MU_BLAS, 2)
        want = C.oracle_blas(op, np.ascontiguousarray(a), np.ascontiguousarray(b), C.Q_BLAS, C.MU_BLAS,
                             x=C.AXPY_X)
        assert np.array_equal(c, want), op


def test_uniform_pairs_are_residues():
    x = R.uniform_pairs(3, 100_000, C.Q_NTT)
    q_hi, q_lo = C.Q_NTT >> 64, C.Q_NTT & ((1 << 64) - 1)
    assert (x[:, 0] <= q_hi).all()
    assert not ((x[:, 0] == q_hi) & (x[:, 1] >= q_lo)).any()
    assert x.ctypes.data % 64 == 0


def test_topology_counts():
    t = R.host_topology()
    assert 1 <= t["physical_cores"] <= t["logical_cpus"]
    assert t["smt"] in ("on", "off", "unknown", "notsupported", "forceoff", "notimplemented")
    assert R.thread_choices(t)[0] == t["logical_cpus"]


@needs_ref
def test_reference_arm_is_clean_and_like_for_like():
    code = ("import runpy, sys, json\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1']\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = [l.split()[-1] for l in open('/proc/self/maps') if '.so' in l]\n"
            "print(json.dumps({'so': sorted(set(maps))}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600, check=True).stdout.strip().splitlines()
    line = json.loads(out[0])
    so = json.loads(out[-1])["so"]
    assert not any("libbntt" in p for p in so), "the reference arm loaded the product library"
    assert any("oracle/_ref/libref_ntt_" in p for p in so)
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["config"] == bench.workload_config(1)
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == cb["threads"] >= 1
    assert cb["physical_cores"] >= 1 and cb["smt"]
    assert cb["full_sequence"]["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]

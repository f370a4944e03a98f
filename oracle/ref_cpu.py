"""The reference's own CPU code, timed on this host's cores (bench.py's CPU
baseline and its reference arm).

TEST / MEASUREMENT INFRASTRUCTURE ONLY.  It drives the benchNTT functions
that oracle/Makefile compiles from the reference's sources into oracle/_ref/
(ref_harness.c entry points, ref_batch.c job runner) and never loads the
product library: inputs are generated with numpy here.

NTT: a whole mixed-size job list runs in one parallel run per measurement
(threads take same-size runs of transforms from a shared counter, largest
first), in two forms:
  ntt_only  ntt() alone per transform, each size's table expanded once
            beforehand: the region the reference drivers time
            (src/ntt_avx512.c:583-590, src/ntt_avx2.c:713-718,
            src/ntt_scalar.c:670-676);
  full      the whole per-call sequence per transform (ntt_pre + ntt +
            ntt_post for the SIMD builds, src/ntt_avx512.c:581-594).
BLAS: the reference's fixed-length (1024) vector functions applied chunk by
chunk over the whole vector on all threads (src/blas_avx512.c:401-476).
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
M64 = (1 << 64) - 1


# ------------------------------------------------------------------ host
def host_topology() -> dict:
    """Logical CPUs this process may use, the physical cores behind them and
    the SMT state (Linux sysfs)."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    cores = set()
    for c in cpus:
        base = f"/sys/devices/system/cpu/cpu{c}/topology"
        try:
            core = open(f"{base}/core_id").read().strip()
            pkg = open(f"{base}/physical_package_id").read().strip()
            cores.add((pkg, core))
        except OSError:
            cores.add(("?", str(c)))
    try:
        smt = open("/sys/devices/system/cpu/smt/active").read().strip()
        smt = {"1": "on", "0": "off"}.get(smt, smt)
    except OSError:
        smt = "unknown"
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"logical_cpus": len(cpus), "physical_cores": len(cores), "smt": smt, "model": model}


def cpu_flags() -> set:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def best_impl() -> str | None:
    """The reference's fastest build this host runs (AVX-512, else AVX2,
    else scalar), or None when oracle/_ref has not been built."""
    flags = cpu_flags()
    for impl, need in (("avx512", ("avx512f", "avx512dq")), ("avx2", ("avx2",)), ("scalar", ())):
        if all(f in flags for f in need) and os.path.exists(os.path.join(REF_DIR, f"libref_ntt_{impl}_10.so")):
            return impl
    return None


# ----------------------------------------------------------------- inputs
def uniform_pairs(seed: int, count: int, q: int) -> np.ndarray:
    """`count` residues uniform in [0, q) (q = 2^124 - k, k < 2^64) as
    hi-first u64 pairs, 64-byte aligned.  The rare draws at or above q
    (probability below 2^-100) are folded back below q."""
    rng = np.random.default_rng(seed)
    out = aligned_pairs(count)
    qh, ql = q >> 64, q & M64
    out[:, 0] = rng.integers(0, qh + 1, size=count, dtype=np.uint64)
    out[:, 1] = rng.integers(0, M64, size=count, dtype=np.uint64, endpoint=True)
    top = (out[:, 0] == qh) & (out[:, 1] >= ql)
    out[top, 1] -= np.uint64(ql)
    return out


def aligned_pairs(count: int) -> np.ndarray:
    """An uninitialised (count, 2) uint64 array starting on a 64-byte boundary
    (the SIMD reference loads whole vectors with aligned instructions)."""
    raw = np.empty(count * 2 + 8, dtype=np.uint64)
    off = (-raw.ctypes.data % 64) // 8
    return raw[off:off + count * 2].reshape(count, 2)


# -------------------------------------------------------------------- NTT
class RefSizeC(ctypes.Structure):
    _fields_ = [("scratch_new", ctypes.c_void_p), ("scratch_free", ctypes.c_void_p),
                ("ntt_only", ctypes.c_void_p), ("ntt_full", ctypes.c_void_p),
                ("prep", ctypes.c_void_p), ("T", ctypes.c_void_p)]


class RefTaskC(ctypes.Structure):
    _fields_ = [("log2n", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("x", ctypes.c_void_p), ("y", ctypes.c_void_p)]


MAX_LOG2N = 24


class RefNttBatch:
    """One job list (sizes `logns`), laid out largest size first, with the
    reference's per-size functions and tables, ready to time."""

    def __init__(self, logns, q: int, mu: int, table_seed_base: int, input_seed: int,
                 impl: str | None = None, elems_per_task: int = 8192):
        self.impl = impl or best_impl()
        if self.impl is None:
            raise RuntimeError("oracle/_ref is not built (make -C oracle ref)")
        self.q, self.mu = q, mu
        logns = np.sort(np.asarray(logns, dtype=np.int64))[::-1]
        self.count = len(logns)
        self.total = int(np.sum(np.left_shift(1, logns)))
        self.x = uniform_pairs(input_seed, self.total, q)
        self.y = aligned_pairs(self.total)
        if self.impl == "scalar":   # the scalar ntt() reads native uint128_t arrays
            self.x_native = aligned_pairs(self.total)
            self.x_native[:, 0], self.x_native[:, 1] = self.x[:, 1], self.x[:, 0]
        self.runner = ctypes.CDLL(os.path.join(REF_DIR, "libref_batch.so"))
        self.runner.bntt_ref_run_tasks.restype = ctypes.c_double
        self.runner.bntt_ref_run_tasks.argtypes = [ctypes.POINTER(RefSizeC), ctypes.POINTER(RefTaskC),
                                                    ctypes.c_size_t, ctypes.c_int] + \
            [ctypes.c_uint64] * 4 + [ctypes.c_int]
        self.libs, self.tables, self.preps = {}, {}, {}
        self.sizes = (RefSizeC * (MAX_LOG2N + 1))()
        qm = (q >> 64, q & M64, mu >> 64, mu & M64)
        for n in sorted(set(int(v) for v in logns)):
            lib = ctypes.CDLL(os.path.join(REF_DIR, f"libref_ntt_{self.impl}_{n}.so"))
            lib.bntt_ref_prep.restype = ctypes.c_void_p
            lib.bntt_ref_prep.argtypes = [ctypes.c_void_p] + [ctypes.c_uint64] * 4
            lib.bntt_ref_prep_free.argtypes = [ctypes.c_void_p]
            lib.bntt_ref_init()
            t = uniform_pairs(table_seed_base + n, 1 << n, q)
            self.libs[n], self.tables[n] = lib, t
            self.preps[n] = lib.bntt_ref_prep(t.ctypes.data, *qm)   # table expansion, untimed
            s = self.sizes[n]
            s.scratch_new = ctypes.cast(lib.bntt_ref_scratch_new, ctypes.c_void_p).value
            s.scratch_free = ctypes.cast(lib.bntt_ref_scratch_free, ctypes.c_void_p).value
            s.ntt_only = ctypes.cast(lib.bntt_ref_ntt_only, ctypes.c_void_p).value
            s.ntt_full = ctypes.cast(lib.bntt_ref_ntt_full, ctypes.c_void_p).value
            s.prep = self.preps[n]
            s.T = t.ctypes.data
        # tasks: runs of same-size transforms of about elems_per_task elements
        tasks = []
        pos = 0
        i = 0
        while i < len(logns):
            n = int(logns[i])
            j = i
            per = max(1, elems_per_task >> n)
            while j < len(logns) and logns[j] == n and j - i < per:
                j += 1
            tasks.append((n, j - i, pos))
            pos += (j - i) << n
            i = j
        self.tasks = (RefTaskC * len(tasks))()
        for k, (n, c, p) in enumerate(tasks):
            self.tasks[k].log2n, self.tasks[k].count = n, c
            self.tasks[k].y = self.y.ctypes.data + p * 16
        self._xbase = {"full": self.x.ctypes.data,
                       "ntt_only": (self.x_native if self.impl == "scalar" else self.x).ctypes.data}
        self._offsets = [p for _, _, p in tasks]
        self.qm = qm

    def run(self, mode: str, threads: int) -> float:
        """Seconds for the whole job list on `threads` threads."""
        base = self._xbase[mode]
        for k, p in enumerate(self._offsets):
            self.tasks[k].x = base + p * 16
        t = self.runner.bntt_ref_run_tasks(self.sizes, self.tasks, len(self.tasks),
                                           0 if mode == "ntt_only" else 1, *self.qm, threads)
        if t < 0:
            raise RuntimeError("reference job runner refused the task list")
        return t

    def close(self) -> None:
        for n, p in self.preps.items():
            self.libs[n].bntt_ref_prep_free(p)
        self.preps.clear()


def thread_choices(topo: dict) -> list[int]:
    """One thread per logical CPU, and one per physical core when SMT gives
    more logical CPUs than cores."""
    out = [topo["logical_cpus"]]
    if 0 < topo["physical_cores"] < topo["logical_cpus"]:
        out.append(topo["physical_cores"])
    return out


# ------------------------------------------------------------------- BLAS
class RefBlas:
    """The reference's vector functions over long vectors (chunks of 1024)."""

    OPS = {"vvadd": 0, "vvsub": 1, "vvmul": 2, "axpy": 3}

    def __init__(self, impl: str | None = None):
        flags = cpu_flags()
        if impl is None:
            for cand, need in (("avx512", ("avx512f", "avx512dq")), ("avx2", ("avx2",)), ("scalar", ())):
                if all(f in flags for f in need) and \
                        os.path.exists(os.path.join(REF_DIR, f"libref_blas_{cand}.so")):
                    impl = cand
                    break
        if impl is None:
            raise RuntimeError("oracle/_ref is not built (make -C oracle ref)")
        self.impl = impl
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, f"libref_blas_{impl}.so"))
        self.lib.bntt_ref_blas.restype = ctypes.c_double
        self.lib.bntt_ref_blas.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + \
            [ctypes.c_uint64] * 2 + [ctypes.c_size_t] + [ctypes.c_uint64] * 4 + [ctypes.c_int]

    def run(self, op: str, c: np.ndarray, a: np.ndarray, b: np.ndarray, x: int, q: int, mu: int,
            threads: int) -> float:
        t = self.lib.bntt_ref_blas(self.OPS[op], c.ctypes.data, a.ctypes.data, b.ctypes.data,
                                   x >> 64, x & M64, a.shape[0], q >> 64, q & M64, mu >> 64, mu & M64,
                                   threads)
        if t < 0:
            raise RuntimeError("length must be a multiple of 1024")
        return t


def time_call(fn, reps: int) -> list[float]:
    out = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        out.append(time.perf_counter() - t0)
    return out

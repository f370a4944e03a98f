"""Benchmark of the benchNTT hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (one "step"): the uneven batch -- 100,000 forward 128-bit
NTTs with N log-uniform over 2^4..2^10 plus 64 at 2^16 and 4 at 2^20 (modulus
2^124 - 719 of the reference NTT drivers), run by one graph launch of the
persistent work-queue kernel.  `value` is transforms per second with inputs
resident in HBM; `e2e` is the same metric from pinned host buffers, every
step one bntt_batch_run_host_async call (all inputs copied in, all outputs
copied out) queued back to back with one bntt_batch_sync at the end, and
beside it one synchronous bntt_batch_run_host per step.  The same line
carries a new job list every step, the inverse batch, the per-call GPU path
on the same jobs, the BLAS ops at 2^24
elements in GB/s, uniform batches of 65,536 transforms per size, the roofline
of the persistent kernel against the measured IMAD pipe peak, the reference's
CPU throughput on the same workload (timed on this host's cores), and the SM
clocks sampled during the timed region.

Under torchrun (N > 1) every rank runs the same per-GPU batch on its own GPU
(no data exchange: the transforms are independent), the timed region is
bracketed by barriers and the slowest rank's time is used.

--impl reference times the reference's own CPU implementation (AVX-512 build
when the host has it, else AVX2, else scalar; compiled from the benchNTT
sources into oracle/_ref) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched 128b NTT/s and BLAS GB/s vs per-call GPU path; bit-exact; p99 latency"
UNIT = "NTT/s"
Q_NTT = (1152921504606846975 << 64) | 18446744073709550897
MU_NTT = (9223372036854775808 << 64) | 5752
Q_BLAS = (0x0FFFFFFFFFFFFFFF << 64) | 0xFFFFFFFFFFFFFFC5
MU_BLAS = (0x8000000000000000 << 64) | 0x1D8
AXPY_X = (208488538572646751 << 64) | 12808410693871070164
IMAD_PER_BUTTERFLY = 80      # generic 32-bit-limb Barrett mulmod (algorithmic count)
HBM_BYTES_PER_ELEM_BLAS = 48  # two 16-byte reads and one write


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the uneven batch (profiling captures of a smaller case)")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the persistent-kernel step (for profiler launch lists)")
    ap.add_argument("--only", choices=["uniform", "inverse", "inverse_batch", "blas", "serving"], default=None,
                    help="run one secondary benchmark alone (profiling captures)")
    ap.add_argument("--logn", type=int, default=10, help="size for --only uniform")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (profiling captures: no tuning launches first)")
    return ap.parse_args()


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons polled through NVML (read only)
    every ~5 ms while the timed region runs."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.thread = None
        self.stop_flag = False
        self.err = None

    def _poll(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.device]) if vis else self.device
            h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            while not self.stop_flag:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetPowerUsage(h) / 1000.0, int(get_reasons(h))))
                time.sleep(0.005)
            nv.nvmlShutdown()
        except Exception as e:  # NVML missing: report, do not fail the benchmark
            self.err = repr(e)

    def start(self):
        import threading
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        time.sleep(0.05)

    def stop(self) -> dict:
        self.stop_flag = True
        if self.thread:
            self.thread.join()
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "error": self.err}
        peak_p = max(p for _, p, _ in self.samples)
        loaded = [s for s in self.samples if s[1] >= 0.6 * peak_p] or self.samples
        reasons = sorted({name for _, _, r in loaded for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(c for c, _, _ in loaded), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples),
                "samples_under_load": len(loaded), "power_w_max": peak_p, "source": "NVML"}


# ---------------------------------------------------------------- CPU side
def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def ref_impl() -> tuple[str, str]:
    """(implementation, kind) of the CPU baseline available on this host."""
    flags = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags = line
                break
    except OSError:
        pass
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    for impl, need in (("avx512", ("avx512f", "avx512dq")), ("avx2", ("avx2",)), ("scalar", ())):
        if all(f in flags.split() for f in need) and \
                os.path.exists(os.path.join(ref_dir, f"libref_ntt_{impl}_10.so")):
            return impl, "reference"
    return "oracle", "port"


class CpuNtt:
    """The reference's per-size NTT functions (or the oracle restatement)."""

    def __init__(self):
        self.impl, self.kind = ref_impl()
        self.libs = {}

    def lib(self, logn: int):
        if logn not in self.libs:
            if self.kind == "reference":
                l = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref",
                                             f"libref_ntt_{self.impl}_{logn}.so"))
                l.bntt_ref_ntt_batch.restype = ctypes.c_double
                l.bntt_ref_ntt_batch.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_size_t] + \
                    [ctypes.c_uint64] * 4 + [ctypes.c_int]
            else:
                path = os.path.join(ROOT, "oracle", "liboracle.so")
                if not os.path.exists(path):
                    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"],
                                   check=True, stdout=subprocess.DEVNULL)
                l = ctypes.CDLL(path)
                l.orc_ntt_batch.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_size_t] + \
                    [ctypes.c_uint64] * 4 + [ctypes.c_int, ctypes.c_int]
            self.libs[logn] = l
        return self.libs[logn]

    def run(self, logn, y, x, t, count, threads) -> float:
        """Seconds for `count` transforms of size 2^logn on `threads` threads."""
        l = self.lib(logn)
        args = (y.ctypes.data, x.ctypes.data, t.ctypes.data)
        qm = (Q_NTT >> 64, Q_NTT & (2**64 - 1), MU_NTT >> 64, MU_NTT & (2**64 - 1))
        if self.kind == "reference":
            return l.bntt_ref_ntt_batch(*args, count, *qm, threads)
        t0 = time.perf_counter()
        l.orc_ntt_batch(y.ctypes.data, x.ctypes.data, t.ctypes.data, logn, count, *qm, 0, threads)
        return time.perf_counter() - t0


def cpu_uneven_throughput(batch, budget_s: float, threads: int, cpu: CpuNtt = None) -> dict:
    """Reference throughput on the uneven batch from a bounded, stratified
    sample: per size, a sample of transforms run on all threads gives the
    per-transform CPU cost c_N (thread-seconds); the batch then needs
    max(sum(count_N * c_N) / threads, max c_N) seconds with perfect packing."""
    import benchntt_b200 as bn
    cpu = cpu or CpuNtt()
    counts = {int(n): int((batch.logns == n).sum()) for n in batch.sizes}
    cost = {}
    per_size = budget_s / len(counts)
    for n, cnt in sorted(counts.items()):
        size = 1 << n
        t = bn.fill_uniform(2000 + n, size, Q_NTT)
        k = min(cnt, max(1, threads))
        k_max = max(k, min(cnt, int(2e8 // (16 * size))))
        xs = bn.fill_uniform(11, size * k_max, Q_NTT)
        y = np.empty_like(xs)
        used = min(threads, k)
        dt = cpu.run(n, y, xs, t, k, used)          # first pass sizes the sample
        reps = k
        while dt < per_size * 0.5 and reps < k_max:
            reps = min(k_max, max(reps * 2, int(reps * per_size / max(dt, 1e-6) * 0.5)))
            used = min(threads, reps)
            dt = cpu.run(n, y[: reps * size], xs[: reps * size], t, reps, used)
        cost[n] = dt * used / reps
    work = sum(counts[n] * cost[n] for n in counts)
    t_batch = max(work / threads, max(cost.values()))
    return {"value": batch.count / t_batch, "unit": UNIT, "cores": threads, "kind": cpu.kind,
            "impl": cpu.impl,
            "sample": ("stratified: per size, a timed sample of transforms on all threads "
                       "gives the per-transform CPU cost; batch time = max(sum(count*cost)/cores, "
                       "max cost); sample budget %.0f s" % budget_s),
            "seconds_per_transform": {str(1 << n): cost[n] for n in sorted(cost)},
            "batch_seconds": t_batch}


# ------------------------------------------------------------- GPU helpers
def cuda_events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def profiles_traffic(name: str):
    """traffic_bytes_per_launch recorded in profiles/<name>.md (ncu capture)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except (OSError, ValueError):
        return None
    return None


def run_only(args, dist: Dist):
    """One secondary benchmark on its own (for ncu captures of one kernel)."""
    import torch

    import benchntt_b200 as bn
    dev = dist.local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = bn.Context(dev, stream=stream.cuda_stream)
    if args.only in ("uniform", "inverse"):
        res = uniform_bench(args, ctx, stream, ctx.imad_peak(), sizes=[args.logn],
                            inverse=args.only == "inverse")
    elif args.only == "serving":
        res = serving_bench(args, ctx)
    elif args.only == "inverse_batch":
        res = inverse_batch_only(args, ctx, stream)
    else:
        res = blas_bench(args, ctx, stream, measured_peaks())
    return {"only": args.only, "result": res}, ctx


def run_ours(args, dist: Dist):
    import torch

    import benchntt_b200 as bn
    from benchntt_b200 import workloads as W

    dev = dist.local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = bn.Context(dev, stream=stream.cuda_stream)
    L = bn.lib()

    # ------------------------------------------------------------ autotuner
    import tempfile
    tune_path = os.path.join(tempfile.mkdtemp(), "bntt.tune")
    t_tune = time.perf_counter()
    tuned = []
    if not args.no_tune:
        ctx.autotune(tune_path)
        tuned = [l.strip() for l in open(tune_path) if l.startswith(("sub ", "batch "))]
    tune_s = time.perf_counter() - t_tune

    # ---------------------------------------------------- headline workload
    batch = W.uneven_batch()
    if args.scale < 1.0:
        n_small = max(1, int(100_000 * args.scale))
        large = tuple((l, max(1, int(c * args.scale))) for l, c in ((16, 64), (20, 4)))
        batch = W.uneven_batch(n_small=n_small, large=large)
    mod = bn.modulus(Q_NTT, MU_NTT)
    plans = {n: bn.Plan(ctx, n, Q_NTT, MU_NTT,
                        bn.fill_uniform(W.SEED_TWIDDLE_BASE + n, 1 << n, Q_NTT))
             for n in batch.sizes}
    pid = {n: i for i, n in enumerate(batch.sizes)}
    x = torch.empty((batch.total, 2), dtype=torch.int64, device=dev)
    y = torch.empty_like(x)
    # each rank transforms its own inputs (weak scaling: same work per GPU)
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), batch.total, W.SEED_INPUT + dist.rank,
                                     0, ctypes.byref(mod), 0))
    engine = bn.Batch(ctx, [plans[n] for n in batch.sizes])
    offs = batch.offsets * 16
    jobs = bn.Batch.jobs([x.data_ptr() + int(o) for o in offs], [y.data_ptr() + int(o) for o in offs],
                         [pid[int(n)] for n in batch.logns])
    for _ in range(args.warmup):
        engine.run_dev(jobs)
    ctx.synchronize()
    if engine.status() != bn.OK:
        raise RuntimeError("batch kernel reported a timed-out wait")
    clocks = ClockSampler(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    e0, e1 = cuda_events()
    e0.record(stream)
    for _ in range(args.steps):
        engine.run_dev(jobs)
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    gpu_launches = ctx.launches - launches0
    ms_local = e0.elapsed_time(e1) / args.steps
    ms = dist.max(ms_local)
    value = batch.count * dist.world / (ms * 1e-3)

    # roofline of the persistent kernel (one launch per step)
    bfly = batch.butterflies
    imad_peak = ctx.imad_peak()
    achieved = IMAD_PER_BUTTERFLY * bfly / (ms_local * 1e-3)
    alg_bytes = 32.0 * batch.total      # read every input, write every output once
    traffic = profiles_traffic("k_batch_uneven.md")
    if traffic is not None and args.scale < 1.0:
        traffic = None
    peaks = measured_peaks()
    roofline = {
        "bound": "imad", "kernel": "k_batch (persistent work queue)",
        "achieved": achieved / 1e12, "peak": imad_peak / 1e12, "unit": "T IMAD-op/s",
        "frac": achieved / imad_peak, "peak_source": "measured live: bntt_probe_imad_peak",
        "algorithmic": f"{IMAD_PER_BUTTERFLY} IMAD per butterfly x {bfly} butterflies per launch",
        "traffic": traffic,
        "butterfly_ceiling": butterfly_ceiling(ctx, bfly, ms_local),
        "hbm": {"achieved_gbs": alg_bytes / (ms_local * 1e-3) / 1e9,
                "peak_gbs": peaks.get("hbm_gbs"), "algorithmic_bytes": alg_bytes,
                "frac": (alg_bytes / (ms_local * 1e-3) / 1e9) / peaks["hbm_gbs"]
                if peaks.get("hbm_gbs") else None,
                "peak_source": "MEASURED_PEAKS.json" if peaks.get("from_file") else "fallback"},
    }

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u128 (4 x u32 limbs, exact integer)",
        "data": "synthetic: seeded uniform residues in [0, q) and seeded per-size twiddle tables",
        "config": {"workload": "uneven_batch", "transforms": batch.count,
                   "sizes": "100,000 x N=2^4..2^10 (log-uniform) + 64 x 2^16 + 4 x 2^20"
                   if args.scale == 1.0 else f"scaled x{args.scale}",
                   "modulus": "2^124-719 (src/ntt_scalar.c:633)",
                   "l2": f"inputs {batch.total * 16 / 1e6:.0f} MB > 126 MB L2 (no flush needed)",
                   "parallelism": f"independent batch per GPU x{dist.world}",
                   "launch": "one CUDA-graph launch of the persistent kernel per step"},
        "gpu_launches": gpu_launches,
        "roofline": roofline,
        "clocks": clk,
        "parity": "bit-exact vs the reference: tests/test_gpu_batch.py::test_full_uneven_batch_matches_oracle",
        "autotune": {"seconds": tune_s, "choices": tuned,
                     "format": "sub m map fast logr tpc minb | batch m logr tpc"},
    }
    if args.headline_only:
        return result, ctx

    # ------------------------------------------------------------ e2e (host)
    result["e2e"] = e2e_uneven(args, dist, ctx, engine, batch, pid)
    # ------------------------------------------- a new job list every step
    result["new_job_list_each_step"] = fresh_lists(args, ctx, stream, engine, jobs, batch, value)
    # ---------------------------------------------------------- per-call path
    result["per_call"] = per_call(args, dist, ctx, stream, engine, jobs, batch, value)
    # ------------------------------------- one transform of N = 1024 per call
    result["single_ntt_1024"] = single_ntt(args, ctx, stream)
    # ----------------------------------------------------------------- BLAS
    result["blas"] = blas_bench(args, ctx, stream, peaks)
    # --------------------------------------------------------- uniform sizes
    result["uniform"] = uniform_bench(args, ctx, stream, imad_peak)
    # ------------------------------------- inverse of the same batch, one launch
    result["inverse_batch"] = inverse_batch_bench(args, ctx, stream, engine, jobs, batch, value)
    # --------------------------------- fused transform + pointwise product
    result["fused_mul"] = fused_bench(args, ctx, stream)
    # ------------------------------------------- NTT-friendly prime (negacyclic)
    result["negacyclic"] = negacyclic_bench(args, ctx, stream, batch, value)
    # ------------------------------- inverse transform and polynomial products
    result["polymul"] = polymul_bench(args, ctx, stream)
    # --------------------------------------------------------------- serving
    engine.close()
    del x, y
    result["serving"] = serving_bench(args, ctx)
    for p in plans.values():
        p.close()
    return result, ctx


def butterfly_ceiling(ctx, bfly: int, ms: float) -> dict:
    """The kernel's butterfly rate against the same butterfly on registers
    (no memory, no index arithmetic) at the same occupancy."""
    peak = ctx.butterfly_peak()
    achieved = bfly / (ms * 1e-3)
    return {"achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "G butterflies/s",
            "frac": achieved / peak, "peak_source": "measured live: bntt_probe_butterfly_peak"}


def measured_peaks() -> dict:
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        d["from_file"] = True
        return d
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "from_file": False}


def e2e_uneven(args, dist, ctx, engine, batch, pid) -> dict:
    """The uneven batch from pinned host buffers: every step copies all
    inputs in and all outputs out (queued steps, and one call at a time)."""
    import torch

    import benchntt_b200 as bn
    xh = torch.empty((batch.total, 2), dtype=torch.int64, pin_memory=True)
    yh = torch.empty_like(xh, pin_memory=True)
    L = bn.lib()
    mod = bn.modulus(Q_NTT, MU_NTT)
    bn.check(L.bntt_fill_uniform_host(xh.data_ptr(), batch.total, 11, 0, ctypes.byref(mod), 0))
    offs = batch.offsets * 16
    hjobs = bn.Batch.jobs([xh.data_ptr() + int(o) for o in offs],
                          [yh.data_ptr() + int(o) for o in offs], [pid[int(n)] for n in batch.logns])
    steps = max(3, min(args.steps, 10))

    def timed(queued: bool) -> float:
        # queued: every step is one bntt_batch_run_host_async call, the steps
        # back to back and one bntt_batch_sync at the end (a stream of
        # batches); otherwise one synchronous bntt_batch_run_host per step
        for _ in range(max(1, min(args.warmup, 3))):
            engine.run_host_async(hjobs) if queued else engine.run_host(hjobs)
        engine.sync()
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            engine.run_host_async(hjobs) if queued else engine.run_host(hjobs)
        engine.sync()
        return dist.max((time.perf_counter() - t0) / steps)

    dt = timed(True)
    dt_sync = timed(False)
    nbytes = batch.total * 16
    link = pcie_both_ways(xh, yh)
    del xh, yh
    return {"value": batch.count * dist.world / dt, "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "ms_per_step": dt * 1e3, "steps": steps,
            "api": "bntt_batch_run_host_async per step, back to back, then bntt_batch_sync "
                   "(pinned host buffers; every step copies all inputs in and all outputs out)",
            "one_call_at_a_time": {"value": batch.count * dist.world / dt_sync, "ms_per_step": dt_sync * 1e3,
                                   "api": "bntt_batch_run_host (synchronous) per step"},
            "pcie_gbs_each_way": nbytes / dt / 1e9,
            "pcie_peak_gbs_each_way": link,
            "pcie_frac": (nbytes / dt / 1e9) / link if link else None,
            "pcie_peak_source": "measured live: concurrent pinned H2D and D2H copies of the same buffers"}


def pcie_both_ways(xh, yh) -> float:
    """GB/s each way of plain concurrent pinned copies (H2D of xh, D2H into
    yh): the link bound of the host path."""
    import torch
    dx = torch.empty_like(xh, device="cuda")
    dy = torch.empty_like(yh, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def both():
        with torch.cuda.stream(s1):
            dx.copy_(xh, non_blocking=True)
        with torch.cuda.stream(s2):
            yh.copy_(dy, non_blocking=True)

    both()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        both()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / 3
    del dx, dy
    return xh.numel() * 8 / dt / 1e9


def single_ntt(args, ctx, stream, logn: int = 10) -> dict:
    """One forward NTT of N = 1024 per call, the reference programs' unit of
    work (src/ntt_scalar.c:582): the plain one-launch device path (calls back
    to back on one stream, and one call with the host waiting for it), and the
    host call that copies the input in and the output out (plan cached)."""
    import torch

    import benchntt_b200 as bn
    from benchntt_b200 import workloads as W
    L = bn.lib()
    n = 1 << logn
    plan = bn.Plan(ctx, logn, Q_NTT, MU_NTT, bn.fill_uniform(W.SEED_TWIDDLE_BASE + logn, n, Q_NTT))
    x = torch.empty((n, 2), dtype=torch.int64, device=ctx.device)
    y = torch.empty_like(x)
    mod = bn.modulus(Q_NTT, MU_NTT)
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), n, 5, 0, ctypes.byref(mod), 0))
    for _ in range(20):
        plan.forward(y, x, 1)
    torch.cuda.synchronize()
    reps = 200
    e0, e1 = cuda_events()
    e0.record(stream)
    for _ in range(reps):
        plan.forward(y, x, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    back_to_back_us = e0.elapsed_time(e1) / reps * 1e3
    t0 = time.perf_counter()
    for _ in range(reps):
        plan.forward(y, x, 1)
        torch.cuda.synchronize()
    sync_us = (time.perf_counter() - t0) / reps * 1e6
    xh = bn.fill_uniform(5, n, Q_NTT)
    yh = np.empty_like(xh)
    for _ in range(10):
        plan.forward(yh, xh)
    t0 = time.perf_counter()
    for _ in range(reps):
        plan.forward(yh, xh)
    host_us = (time.perf_counter() - t0) / reps * 1e6
    plan.close()
    return {"n": n, "device_us_per_call_back_to_back": back_to_back_us,
            "device_us_per_call_waited": sync_us, "host_buffers_us_per_call": host_us,
            "api": "bntt_ntt_forward_dev / bntt_ntt_forward_host, batch = 1"}


def fresh_lists(args, ctx, stream, engine, jobs, batch, batched_value) -> dict:
    """The headline batch with the job list alternating between two orders
    (the given one and its reverse), so every step is a job list the engine
    did not run last: schedule built on the host, copied while the previous
    launch runs, launched without a graph."""
    import torch

    import benchntt_b200 as bn
    rev = (bn.JobC * len(jobs))(*reversed(list(jobs)))
    lists = (jobs, rev)
    for i in range(4):
        engine.run_dev(lists[i % 2])
    ctx.synchronize()
    steps = max(10, min(args.steps, 40))
    e0, e1 = cuda_events()
    t0 = time.perf_counter()
    e0.record(stream)
    for i in range(steps):
        engine.run_dev(lists[i % 2])
    e1.record(stream)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / steps
    ms = e0.elapsed_time(e1) / steps
    return {"value": batch.count / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "host_wall_ms_per_step": wall * 1e3, "vs_same_list": batch.count / (ms * 1e-3) / batched_value}


def per_call(args, dist, ctx, stream, engine, jobs, batch, batched_value) -> dict:
    """The same jobs, one launch per transform (per HBM pass above 2^10)."""
    import torch
    engine.run_percall_dev(jobs)   # warm-up pass
    ctx.synchronize()
    launches = 0
    e0, e1 = cuda_events()
    reps = 2
    e0.record(stream)
    for _ in range(reps):
        engine.run_percall_dev(jobs)
        launches += engine.last_launches
    e1.record(stream)
    torch.cuda.synchronize()
    ms = dist.max(e0.elapsed_time(e1) / reps)
    v = batch.count * dist.world / (ms * 1e-3)
    return {"value": v, "unit": UNIT, "ms_per_step": ms, "launches_per_step": launches // reps,
            "batched_over_per_call": batched_value / v}


def blas_bench(args, ctx, stream, peaks) -> dict:
    import torch

    import benchntt_b200 as bn
    L = bn.lib()
    n = 1 << 24
    mod = bn.modulus(Q_BLAS, MU_BLAS)
    a = torch.empty((n, 2), dtype=torch.int64, device=ctx.device)
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, a.data_ptr(), n, 3000, 0, ctypes.byref(mod), 0))
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, b.data_ptr(), n, 4000, 0, ctypes.byref(mod), 0))
    res = {"length": n, "bytes_per_op": HBM_BYTES_PER_ELEM_BLAS * n,
           "peak_gbs": peaks.get("hbm_gbs"),
           "peak_source": "MEASURED_PEAKS.json" if peaks.get("from_file") else "fallback",
           "note": "operands 256 MiB each > L2: no flush needed"}
    for op in ("vvadd", "vvsub", "vvmul", "axpy"):
        fn = getattr(L, f"bntt_{op}_dev")

        def go():
            if op == "axpy":
                bn.check(fn(ctx.handle, c.data_ptr(), a.data_ptr(), b.data_ptr(), bn.U128.of(AXPY_X),
                            n, ctypes.byref(mod), 0))
            else:
                bn.check(fn(ctx.handle, c.data_ptr(), a.data_ptr(), b.data_ptr(), n,
                            ctypes.byref(mod), 0))
        for _ in range(max(1, args.warmup) if args.only else max(3, args.warmup)):
            go()
        e0, e1 = cuda_events()
        reps = max(1, args.steps) if args.only else max(5, args.steps)
        e0.record(stream)
        for _ in range(reps):
            go()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = HBM_BYTES_PER_ELEM_BLAS * n / (ms * 1e-3) / 1e9
        res[op] = {"gbs": gbs, "ms": ms, "frac_of_hbm_peak": gbs / peaks["hbm_gbs"]}
    del a, b, c
    return res


L2_FLUSH_BYTES = 256 << 20   # twice the B200's 126 MB L2


def uniform_bench(args, ctx, stream, imad_peak, sizes=(4, 5, 6, 7, 8, 9, 10, 16, 20),
                  inverse=False) -> dict:
    """65,536 transforms of one size, one launch (config: uniform batch);
    above 2^10 points, 2^26 elements.  inverse=True times the inverse."""
    import torch

    import benchntt_b200 as bn
    L = bn.lib()
    mod = bn.modulus(Q_NTT, MU_NTT)
    res = {}
    for logn in sizes:
        n = 1 << logn
        count = 65536 if logn <= 10 else (1 << 26) >> logn
        x = torch.empty((n * count, 2), dtype=torch.int64, device=ctx.device)
        y = torch.empty_like(x)
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), n * count, 7, 0,
                                         ctypes.byref(mod), 0))
        plan = bn.Plan(ctx, logn, Q_NTT, MU_NTT, bn.fill_uniform(2000 + logn, n, Q_NTT))
        run = (lambda: plan.inverse(y, x, count)) if inverse else (lambda: plan.forward(y, x, count))
        for _ in range(max(1, min(3, args.warmup))):
            run()
        reps = max(1, args.steps // 2) if args.only else max(5, args.steps // 2)
        small = x.numel() * 8 < L2_FLUSH_BYTES
        if small:   # inputs fit in L2: flush it before each timed launch
            flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=ctx.device)
            ms = 0.0
            for _ in range(reps):
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                e0, e1 = cuda_events()
                e0.record(stream)
                run()
                e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
            ms /= reps
            del flush
        else:
            e0, e1 = cuda_events()
            e0.record(stream)
            for _ in range(reps):
                run()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
        bfly = count * (n // 2) * logn
        res[str(n)] = {"ntt_per_s": count / (ms * 1e-3), "ms": ms,
                       "imad80_frac": IMAD_PER_BUTTERFLY * bfly / (ms * 1e-3) / imad_peak,
                       "l2": "flushed before each timed launch" if small else "inputs larger than L2"}
        plan.close()
        del x, y
    return res


def inverse_batch_only(args, ctx, stream) -> dict:
    """The inverse batch alone on the uneven batch (scaled by --scale), for
    profiling k_batch_inv."""
    import torch

    import benchntt_b200 as bn
    from benchntt_b200 import workloads as W
    L = bn.lib()
    batch = W.uneven_batch()
    if args.scale < 1.0:
        large = tuple((l, max(1, int(c * args.scale))) for l, c in ((16, 64), (20, 4)))
        batch = W.uneven_batch(n_small=max(1, int(100_000 * args.scale)), large=large)
    mod = bn.modulus(Q_NTT, MU_NTT)
    plans = {n: bn.Plan(ctx, n, Q_NTT, MU_NTT, bn.fill_uniform(W.SEED_TWIDDLE_BASE + n, 1 << n, Q_NTT))
             for n in batch.sizes}
    pid = {n: i for i, n in enumerate(batch.sizes)}
    x = torch.empty((batch.total, 2), dtype=torch.int64, device=ctx.device)
    y = torch.empty_like(x)
    bn.check(L.bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), batch.total, W.SEED_INPUT, 0,
                                     ctypes.byref(mod), 0))
    engine = bn.Batch(ctx, [plans[n] for n in batch.sizes])
    offs = batch.offsets * 16
    jobs = bn.Batch.jobs([x.data_ptr() + int(o) for o in offs], [y.data_ptr() + int(o) for o in offs],
                         [pid[int(n)] for n in batch.logns])
    res = inverse_batch_bench(args, ctx, stream, engine, jobs, batch, 1.0)
    res.pop("vs_forward")
    res["transforms"] = batch.count
    engine.close()
    for p in plans.values():
        p.close()
    return res


def inverse_batch_bench(args, ctx, stream, engine, jobs, batch, forward_value) -> dict:
    """bntt_batch_run_inverse_dev on the headline job list: the inverse of
    every transform of the uneven batch in one persistent launch."""
    import torch
    for _ in range(max(3, args.warmup)):
        engine.run_inverse_dev(jobs)
    e0, e1 = cuda_events()
    reps = max(5, args.steps // 4)
    e0.record(stream)
    for _ in range(reps):
        engine.run_inverse_dev(jobs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {"value": batch.count / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "vs_forward": batch.count / (ms * 1e-3) / forward_value,
            "parity": "tests/test_gpu_batch.py::test_inverse_batch_matches_oracle"}


def fused_bench(args, ctx, stream, sizes=(4, 7, 10, 16)) -> dict:
    """y = vector_mul(ntt(x), b) for 2^26 elements per size: the fused call
    (bntt_ntt_forward_mul_dev) against the transform followed by vvmul."""
    import torch

    import benchntt_b200 as bn
    L = bn.lib()
    mod = bn.modulus(Q_NTT, MU_NTT)
    res = {}
    total = 1 << 26
    for logn in sizes:
        n = 1 << logn
        count = total // n
        x = torch.empty((total, 2), dtype=torch.int64, device=ctx.device)
        b = torch.empty_like(x)
        y = torch.empty_like(x)
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), total, 7, 0, ctypes.byref(mod), 0))
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, b.data_ptr(), total, 8, 0, ctypes.byref(mod), 0))
        plan = bn.Plan(ctx, logn, Q_NTT, MU_NTT, bn.fill_uniform(2000 + logn, n, Q_NTT))

        def two_step():
            plan.forward(y, x, count)
            bn.check(L.bntt_vvmul_dev(ctx.handle, y.data_ptr(), y.data_ptr(), b.data_ptr(), total,
                                      ctypes.byref(mod), 0))

        def one_step():
            plan.forward_mul(y, x, b, True, count)

        row = {}
        for name, fn in (("ntt_then_vvmul_ms", two_step), ("fused_ms", one_step)):
            for _ in range(3):
                fn()
            e0, e1 = cuda_events()
            reps = max(5, args.steps // 4)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            row[name] = e0.elapsed_time(e1) / reps
        row["speedup"] = row["ntt_then_vvmul_ms"] / row["fused_ms"]
        row["transforms"] = count
        res[str(n)] = row
        plan.close()
        del x, b, y
    return res


def polymul_bench(args, ctx, stream, sizes=(10, 16)) -> dict:
    """Negacyclic products a * b mod (x^N + 1) in the friendly-prime mode, 2^26
    coefficients per operand: forward(b), forward(a) fused with the pointwise
    product, inverse.  Also the inverse transform alone."""
    import torch

    import benchntt_b200 as bn
    L = bn.lib()
    q, mu = bn.ntt_prime(21)
    w = bn.root_of_unity(q, mu, 21)
    mod = bn.modulus(q, mu)
    total = 1 << 26
    res = {"modulus": f"2^124 - {(1 << 124) - q:#x}"}
    for logn in sizes:
        count = total >> logn
        plan = bn.Plan.negacyclic(ctx, logn, q, mu, bn.powmod(q, mu, w, 1 << (21 - logn - 1)))
        a = torch.empty((total, 2), dtype=torch.int64, device=ctx.device)
        b, bh, c = torch.empty_like(a), torch.empty_like(a), torch.empty_like(a)
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, a.data_ptr(), total, 21, 0, ctypes.byref(mod), 0))
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, b.data_ptr(), total, 22, 0, ctypes.byref(mod), 0))

        def product():
            plan.forward(bh, b, count)
            plan.forward_mul(c, a, bh, True, count)
            plan.inverse(c, c, count)

        def inverse_only():
            plan.inverse(c, bh, count)

        row = {"transforms": count}
        for name, fn in (("inverse", inverse_only), ("product", product)):
            for _ in range(3):
                fn()
            e0, e1 = cuda_events()
            reps = max(5, args.steps // 4)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            row[f"{name}_ms"] = ms
            row[f"{name}_per_s"] = count / (ms * 1e-3)
        res[str(1 << logn)] = row
        plan.close()
        del a, b, bh, c
    return res


def negacyclic_bench(args, ctx, stream, batch, headline_value) -> dict:
    """The headline uneven batch in the NTT-friendly prime mode: prime
    2^124 - (62*2^21 - 1) from bntt_ntt_prime, root-power tables generated on
    the device (bntt_plan_create_negacyclic), same persistent kernel."""
    import torch

    import benchntt_b200 as bn
    from benchntt_b200 import workloads as W

    q, mu = bn.ntt_prime(21)
    w = bn.root_of_unity(q, mu, 21)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plans = {n: bn.Plan.negacyclic(ctx, n, q, mu, bn.powmod(q, mu, w, 1 << (21 - n - 1)))
             for n in batch.sizes}
    ctx.synchronize()
    plan_s = time.perf_counter() - t0
    pid = {n: i for i, n in enumerate(batch.sizes)}
    dev = torch.cuda.current_device()
    x = torch.empty((batch.total, 2), dtype=torch.int64, device=dev)
    y = torch.empty_like(x)
    bn.check(bn.lib().bntt_fill_uniform_dev(ctx.handle, x.data_ptr(), batch.total, W.SEED_INPUT, 0,
                                            ctypes.byref(bn.modulus(q, mu)), 0))
    engine = bn.Batch(ctx, [plans[n] for n in batch.sizes])
    offs = batch.offsets * 16
    jobs = bn.Batch.jobs([x.data_ptr() + int(o) for o in offs], [y.data_ptr() + int(o) for o in offs],
                         [pid[int(n)] for n in batch.logns])
    for _ in range(max(3, args.warmup)):
        engine.run_dev(jobs)
    e0, e1 = cuda_events()
    reps = max(5, args.steps // 2)
    e0.record(stream)
    for _ in range(reps):
        engine.run_dev(jobs)
    e1.record(stream)
    torch.cuda.synchronize()
    if engine.status() != bn.OK:
        raise RuntimeError("batch kernel reported a timed-out wait")
    ms = e0.elapsed_time(e1) / reps
    engine.close()
    for p in plans.values():
        p.close()
    return {"modulus": f"2^124 - {(1 << 124) - q:#x} (2^21 | q - 1)", "value": batch.count / (ms * 1e-3),
            "unit": UNIT, "ms_per_step": ms, "vs_reference_modulus": batch.count / (ms * 1e-3) / headline_value,
            "plan_create_s": plan_s, "tables": "T[k] = psi^brv(k), generated on the device",
            "parity": "tests/test_gpu_negacyclic.py (reference ntt() fixtures, 2^2..2^20)"}


def serving_bench(args, ctx) -> dict:
    """Poisson arrivals at 50k requests/s: 70% forward NTTs with N log-uniform
    over 2^4..2^20, 30% vvmul / axpy with length log-uniform over 2^10..2^22,
    device-resident operands, 32 GiB admission budget.  Continuous batching
    versus the same requests served one call at a time."""
    import torch

    import benchntt_b200 as bn
    from benchntt_b200 import workloads as W
    L = bn.lib()
    sizes = list(range(4, 21))
    plans = [bn.Plan(ctx, n, Q_NTT, MU_NTT, bn.fill_uniform(W.SEED_TWIDDLE_BASE + n, 1 << n, Q_NTT))
             for n in sizes]
    mod, modb = bn.modulus(Q_NTT, MU_NTT), bn.modulus(Q_BLAS, MU_BLAS)
    ntt_in = {}
    for n in sizes:     # one resident input per size
        t = torch.empty((1 << n, 2), dtype=torch.int64, device=ctx.device)
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, t.data_ptr(), 1 << n, 100 + n, 0, ctypes.byref(mod), 0))
        ntt_in[n] = t
    blas_in = {}
    for l in range(10, 23):
        a = torch.empty((1 << l, 2), dtype=torch.int64, device=ctx.device)
        b = torch.empty_like(a)
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, a.data_ptr(), 1 << l, 200 + l, 0, ctypes.byref(modb), 0))
        bn.check(L.bntt_fill_uniform_dev(ctx.handle, b.data_ptr(), 1 << l, 300 + l, 0, ctypes.byref(modb), 0))
        blas_in[l] = (a, b)
    count = 20_000
    trace = W.serving_trace(rate=50_000.0, count=count)
    reqs = (bn.RequestC * count)()
    for i, r in enumerate(trace):
        q = reqs[i]
        q.t_arrive, q.tag = r.t_arrive, i
        if r.kind == "ntt":
            q.kind, q.plan, q.x = bn.REQ_NTT, sizes.index(r.log2), ntt_in[r.log2].data_ptr()
        else:
            a, b = blas_in[r.log2]
            q.kind = bn.REQ_VVMUL if r.kind == "vvmul" else bn.REQ_AXPY
            q.len, q.x, q.b, q.scalar = 1 << r.log2, a.data_ptr(), b.data_ptr(), bn.U128.of(AXPY_X)
    out = {"requests": count, "rate_req_s": 50_000, "mix": "70% NTT 2^4..2^20, 30% vvmul/axpy 2^10..2^22",
           "hbm_budget_bytes": 32 << 30}
    srv = bn.Server(ctx, plans, Q_BLAS, MU_BLAS, hbm_budget=32 << 30, slots=4, max_batch=4096)
    warm = (bn.RequestC * 2000)(*reqs[:2000])   # warm-up on the first 2,000 arrivals
    for mode, serial in (("continuous_batching", False), ("one_call_at_a_time", True)):
        srv.replay(warm, serial=serial)
        lat, wall = srv.replay(reqs, serial=serial)
        out[mode] = {"throughput_req_s": count / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                     "p99_ms": float(np.percentile(lat, 99) * 1e3),
                     "mean_ms": float(lat.mean() * 1e3), "wall_s": wall}
    out["stats"] = srv.stats()
    out["p99_speedup"] = out["one_call_at_a_time"]["p99_ms"] / out["continuous_batching"]["p99_ms"]
    srv.close()
    for p in plans:
        p.close()
    return out


# ---------------------------------------------------------- reference arm
def run_reference(args, dist: Dist):
    from benchntt_b200 import workloads as W
    if dist.rank != 0:
        return None
    batch = W.uneven_batch()
    threads = cpu_threads()
    cpu = CpuNtt()
    budget = max(1.0, min(6.0, 150.0 / max(1, args.steps + args.warmup)))
    vals = []
    last = None
    for i in range(args.warmup + args.steps):
        r = cpu_uneven_throughput(batch, budget, threads, cpu)
        if i >= args.warmup:
            vals.append(r["value"])
            last = r
    value = statistics.median(vals)
    last["value"] = value
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * batch.count / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u128 (uint128_t / 2 x u64)",
        "data": "synthetic: seeded uniform residues in [0, q), seeded per-size twiddle tables",
        "config": {"workload": "uneven_batch", "transforms": batch.count,
                   "sizes": "100,000 x N=2^4..2^10 (log-uniform) + 64 x 2^16 + 4 x 2^20",
                   "modulus": "2^124-719 (src/ntt_scalar.c:633)",
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": last,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    from benchntt_b200.dist import Dist
    args = parse()
    dist = Dist()
    try:
        if args.impl == "reference":
            res = run_reference(args, dist)
            if res is not None:
                print(json.dumps(res), flush=True)
            return
        if args.only:
            res, ctx = run_only(args, dist)
            if dist.rank == 0:
                print(json.dumps(res), flush=True)
            ctx.close()
            return
        res, ctx = run_ours(args, dist)
        if dist.rank == 0 and dist.world == 1 and not args.no_cpu and not args.headline_only:
            from benchntt_b200 import workloads as W
            res["cpu_baseline"] = cpu_uneven_throughput(W.uneven_batch(), 12.0, cpu_threads())
            res["gpu_over_cpu"] = res["value"] / res["cpu_baseline"]["value"]
            res["e2e_over_cpu"] = res["e2e"]["value"] / res["cpu_baseline"]["value"]
            # the same CPU sample per size: the reference's throughput on the
            # uniform batches (all cores, one transform per core at a time)
            cores = res["cpu_baseline"]["cores"]
            one = res.get("single_ntt_1024")
            secs = res["cpu_baseline"].get("seconds_per_transform", {}).get("1024")
            if one and secs:   # one core per transform, as the reference programs run
                one["cpu_reference_us_per_transform"] = secs * 1e6
            for n, secs in res["cpu_baseline"].get("seconds_per_transform", {}).items():
                row = res.get("uniform", {}).get(n)
                if row and secs > 0:
                    row["cpu_reference_ntt_per_s"] = cores / secs
                    row["gpu_over_cpu"] = row["ntt_per_s"] / (cores / secs)
        if dist.rank == 0:
            print(json.dumps(res), flush=True)
        ctx.close()
    finally:
        dist.close()


if __name__ == "__main__":
    main()

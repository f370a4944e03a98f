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
    ap.add_argument("--split", action="store_true",
                    help="under torchrun: split one job list over the ranks by cost (strong "
                         "scaling) instead of one whole batch per rank (weak scaling)")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the persistent-kernel step (for profiler launch lists)")
    ap.add_argument("--only", choices=["uniform", "inverse", "inverse_batch", "blas", "serving"], default=None,
                    help="run one secondary benchmark alone (profiling captures)")
    ap.add_argument("--logn", type=int, default=10, help="size for --only uniform")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (profiling captures: no tuning launches first)")
    ap.add_argument("--tune-save", default=None, help="write the autotuner's choices to this file")
    ap.add_argument("--tune-load", default=None,
                    help="install choices saved earlier instead of tuning (profiling captures)")
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
        # the first NVML initialisation of a process can take a few hundred
        # ms: wait for the first sample, so the timed region is covered
        t0 = time.perf_counter()
        while not self.samples and self.err is None and time.perf_counter() - t0 < 5.0:
            time.sleep(0.005)

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
def ref_cpu():
    """oracle/ref_cpu.py: the reference's own CPU code (built into
    oracle/_ref from the benchNTT sources), timed on this host.  It never
    loads libbntt."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cpu as R
    return R


def workload_config(world: int, scale: float = 1.0) -> dict:
    """The headline workload, identical in both arms' JSON lines."""
    return {"workload": "uneven_batch", "transforms": 100_068 if scale == 1.0 else None,
            "sizes": "100,000 x N=2^4..2^10 (log-uniform) + 64 x 2^16 + 4 x 2^20"
            if scale == 1.0 else f"scaled x{scale}",
            "modulus": "2^124-719 (src/ntt_scalar.c:633)",
            "l2": "inputs 600 MB > 126 MB L2 (no flush needed)",
            "parallelism": f"dp{world}: one independent batch per device"}


def cpu_uneven(logns, steps: int, warmup: int, full_steps: int) -> dict:
    """The reference's CPU code on the whole uneven job list, one parallel run
    per step (threads take runs of same-size transforms from a shared counter,
    largest first), in its own timed form -- ntt() per transform with each
    size's table expanded once beforehand (src/ntt_avx512.c:583-590) -- and
    as the whole per-call sequence (ntt_pre + ntt + ntt_post).  The thread
    count is the faster of one per logical CPU and one per physical core,
    chosen in the warm-up."""
    R = ref_cpu()
    from benchntt_b200 import workloads as W
    topo = R.host_topology()
    rb = R.RefNttBatch(logns, Q_NTT, MU_NTT, W.SEED_TWIDDLE_BASE, W.SEED_INPUT)
    trial = {th: rb.run("ntt_only", th) for th in R.thread_choices(topo)}
    threads = min(trial, key=trial.get)
    for _ in range(max(0, warmup - 1)):
        rb.run("ntt_only", threads)
    only = [rb.run("ntt_only", threads) for _ in range(max(1, steps))]
    rb.run("full", threads)
    full = [rb.run("full", threads) for _ in range(max(1, full_steps))]
    rb.close()
    n = len(logns)
    t_only, t_full = statistics.mean(only), statistics.mean(full)
    return {"value": n / t_only, "unit": UNIT, "cores": threads, "kind": "reference", "impl": rb.impl,
            "threads": threads, "physical_cores": topo["physical_cores"],
            "logical_cpus": topo["logical_cpus"], "smt": topo["smt"], "cpu_model": topo["model"],
            "thread_trials_s": {str(k): v for k, v in trial.items()},
            "timed_region": "ntt() per transform, each size's table expanded once beforehand "
                            "(the reference drivers' timed region, src/ntt_avx512.c:583-590)",
            "sample": f"the whole job list ({n} transforms) per step in one parallel run",
            "ms_per_step": t_only * 1e3, "steps": len(only),
            "full_sequence": {"value": n / t_full, "unit": UNIT, "ms_per_step": t_full * 1e3,
                              "steps": len(full),
                              "timed_region": "ntt_pre + ntt + ntt_post per transform "
                                              "(the reference's whole per-call sequence)"}}


def cpu_extras(threads: int) -> dict:
    """The reference's CPU code on the other configurations: uniform batches
    per size (a sample of each 65,536-transform batch), one transform of
    N = 1024 on one core, and the four vector ops at 2^24 elements."""
    R = ref_cpu()
    from benchntt_b200 import workloads as W
    out = {"uniform": {}, "threads": threads}
    for logn in range(4, 11):
        count = min(65536, (1 << 23) >> logn)
        rb = R.RefNttBatch([logn] * count, Q_NTT, MU_NTT, W.SEED_TWIDDLE_BASE, 7)
        t = min(rb.run("ntt_only", threads) for _ in range(2))
        out["uniform"][str(1 << logn)] = {"ntt_per_s": count / t, "sample_transforms": count}
        rb.close()
    rb = R.RefNttBatch([10] * 256, Q_NTT, MU_NTT, W.SEED_TWIDDLE_BASE, 5)
    t = min(rb.run("ntt_only", 1) for _ in range(3))
    out["single_ntt_1024_us"] = t / 256 * 1e6
    rb.close()
    blas = R.RefBlas()
    n = 1 << 24
    a = R.uniform_pairs(3000, n, Q_BLAS)
    b = R.uniform_pairs(4000, n, Q_BLAS)
    c = R.aligned_pairs(n)
    res = {"impl": blas.impl, "length": n, "threads": threads}
    for op in ("vvadd", "vvsub", "vvmul", "axpy"):
        blas.run(op, c, a, b, AXPY_X, Q_BLAS, MU_BLAS, threads)
        t = min(blas.run(op, c, a, b, AXPY_X, Q_BLAS, MU_BLAS, threads) for _ in range(3))
        res[op] = {"gbs": HBM_BYTES_PER_ELEM_BLAS * n / t / 1e9, "ms": t * 1e3}
    out["blas"] = res
    return out


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
    if args.tune_load:
        ctx.autotune_load(args.tune_load)
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
    if args.tune_load:
        ctx.autotune_load(args.tune_load)
        tuned = [l.strip() for l in open(args.tune_load) if l.startswith(("sub ", "batch "))]
    elif not args.no_tune:
        ctx.autotune(tune_path)
        tuned = [l.strip() for l in open(tune_path) if l.startswith(("sub ", "batch "))]
        if args.tune_save:
            import shutil
            shutil.copy(tune_path, args.tune_save)
    tune_s = time.perf_counter() - t_tune

    # ---------------------------------------------------- headline workload
    batch = W.uneven_batch()
    if args.scale < 1.0:
        n_small = max(1, int(100_000 * args.scale))
        large = tuple((l, max(1, int(c * args.scale))) for l, c in ((16, 64), (20, 4)))
        batch = W.uneven_batch(n_small=n_small, large=large)
    split = args.split and dist.world > 1
    # units of work one step does over the whole job: every rank's batch, or
    # (split) the one job list the ranks share
    units = batch.count if split else batch.count * dist.world
    if split:   # this rank's share of the job list, longest first to the least-loaded rank
        from benchntt_b200.dist import shard_by_cost
        batch = W.make_batch(batch.logns[shard_by_cost(batch.logns, dist.world)[dist.rank]])
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
    value = units / (ms * 1e-3)

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
                "peak_source": peaks["source"]},
    }

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong" if split else "weak", "vs_baseline": None,
        "dtype": "u128 (4 x u32 limbs, exact integer)",
        "data": "synthetic: seeded uniform residues in [0, q) and seeded per-size twiddle tables",
        "config": dict(workload_config(dist.world, args.scale),
                       **({"parallelism": f"dp{dist.world}: one job list split by cost over the devices"}
                          if split else {})),
        "launch": "one CUDA-graph launch of the persistent kernel per step",
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
    result["e2e"] = e2e_uneven(args, dist, ctx, engine, batch, pid, units)
    # ------------------------------------------- a new job list every step
    result["new_job_list_each_step"] = fresh_lists(args, ctx, stream, engine, jobs, batch, value)
    # ---------------------------------------------------------- per-call path
    result["per_call"] = per_call(args, dist, ctx, stream, engine, jobs, units, value)
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


_PEAKS = None


def measured_peaks() -> dict:
    """MEASURED_PEAKS.json when the file is present, else the HBM copy
    bandwidth measured here (a device-to-device copy of 1 GiB, read plus
    write bytes over its time, best of 5)."""
    global _PEAKS
    if _PEAKS is not None:
        return _PEAKS
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        d["from_file"] = True
        d["source"] = "MEASURED_PEAKS.json"
    except (OSError, ValueError):
        d = {"hbm_gbs": live_copy_gbs(), "from_file": False,
             "source": "measured live: device-to-device copy of 1 GiB (read + write bytes)"}
    _PEAKS = d
    return d


def live_copy_gbs() -> float:
    import torch
    a = torch.empty(1 << 30, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    a.fill_(1)
    best = 1e30
    for _ in range(6):
        e0, e1 = cuda_events()
        e0.record()
        b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * (1 << 30) / (best * 1e-3) / 1e9


def e2e_uneven(args, dist, ctx, engine, batch, pid, units: int) -> dict:
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
    return {"value": units / dt, "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "ms_per_step": dt * 1e3, "steps": steps,
            "api": "bntt_batch_run_host_async per step, back to back, then bntt_batch_sync "
                   "(pinned host buffers; every step copies all inputs in and all outputs out)",
            "one_call_at_a_time": {"value": units / dt_sync, "ms_per_step": dt_sync * 1e3,
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
    # the host's own work per new list: the call timed with the device idle
    # (nothing to wait for)
    host = []
    for i in range(6):
        ctx.synchronize()
        t1 = time.perf_counter()
        engine.run_dev(lists[i % 2])
        host.append(time.perf_counter() - t1)
    ctx.synchronize()
    return {"value": batch.count / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "host_wall_ms_per_step": wall * 1e3, "vs_same_list": batch.count / (ms * 1e-3) / batched_value,
            "host_ms_per_new_list": statistics.median(host) * 1e3}


def per_call(args, dist, ctx, stream, engine, jobs, units, batched_value) -> dict:
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
    v = units / (ms * 1e-3)
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
           "peak_source": peaks["source"],
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
    if not args.only:
        res["e2e_note"] = ("e2e_host: bntt_<op>_host from pinned host buffers, both operands copied in and "
                           "the result copied out inside the timed call; GB/s of the op's 48 B per element")
        ah = a.cpu().pin_memory()
        bh = b.cpu().pin_memory()
        ch = torch.empty_like(ah).pin_memory()
        for op in ("vvadd", "vvsub", "vvmul", "axpy"):
            fn = getattr(L, f"bntt_{op}_host")

            def go_host():
                if op == "axpy":
                    bn.check(fn(ctx.handle, ch.data_ptr(), ah.data_ptr(), bh.data_ptr(), bn.U128.of(AXPY_X),
                                n, ctypes.byref(mod), 0))
                else:
                    bn.check(fn(ctx.handle, ch.data_ptr(), ah.data_ptr(), bh.data_ptr(), n,
                                ctypes.byref(mod), 0))
            go_host()
            reps = 3
            t0 = time.perf_counter()
            for _ in range(reps):
                go_host()
            dt = (time.perf_counter() - t0) / reps
            res[op]["e2e_host"] = {"gbs": HBM_BYTES_PER_ELEM_BLAS * n / dt / 1e9, "ms": dt * 1e3,
                                   "h2d_bytes": 32 * n, "d2h_bytes": 16 * n}
        del ah, bh, ch
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
        if logn <= 10 and not inverse and not args.only:
            # the same 65,536 transforms, one launch per transform
            eng = bn.Batch(ctx, [plan])
            base_x, base_y, step = x.data_ptr(), y.data_ptr(), n * 16
            jobs = bn.Batch.jobs([base_x + i * step for i in range(count)],
                                 [base_y + i * step for i in range(count)], [0] * count)
            eng.run_percall_dev(jobs)
            torch.cuda.synchronize()
            e0, e1 = cuda_events()
            e0.record(stream)
            eng.run_percall_dev(jobs)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_pt = e0.elapsed_time(e1)
            row = res[str(n)]
            row["per_transform_ntt_per_s"] = count / (ms_pt * 1e-3)
            row["per_transform_launches"] = eng.last_launches
            row["one_launch_over_per_transform"] = row["ntt_per_s"] / row["per_transform_ntt_per_s"]
            eng.close()
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

    def requests(rate: float):
        trace = W.serving_trace(rate=rate, count=count)
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
        return reqs

    out = {"requests": count, "mix": "70% NTT 2^4..2^20, 30% vvmul/axpy 2^10..2^22",
           "hbm_budget_bytes": 32 << 30,
           "service": "service time = completion - admission (serial: - start of its call)"}
    srv = bn.Server(ctx, plans, Q_BLAS, MU_BLAS, hbm_budget=32 << 30, slots=4, max_batch=4096)

    def replay(rate: float) -> dict:
        reqs = requests(rate)
        warm = (bn.RequestC * 2000)(*reqs[:2000])   # warm-up on the first 2,000 arrivals
        row = {"rate_req_s": rate}
        for mode, serial in (("continuous_batching", False), ("one_call_at_a_time", True)):
            srv.replay(warm, serial=serial)
            lat, svc, wall = srv.replay(reqs, serial=serial, service=True)
            row[mode] = {"throughput_req_s": count / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                         "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                         "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
                         "service_p99_ms": float(np.percentile(svc, 99) * 1e3), "wall_s": wall}
        row["p99_speedup"] = row["one_call_at_a_time"]["p99_ms"] / row["continuous_batching"]["p99_ms"]
        row["service_p99_ratio"] = (row["one_call_at_a_time"]["service_p99_ms"] /
                                    row["continuous_batching"]["service_p99_ms"])
        return row

    out["rate_50k"] = replay(50_000.0)
    out["rate_50k"]["note"] = ("one call at a time cannot sustain 50k req/s: its queue grows through the "
                               "replay, so its latency measures the replay's length")
    # the rate the one-call-at-a-time path sustains: 80 % of its measured throughput
    sustainable = 0.8 * out["rate_50k"]["one_call_at_a_time"]["throughput_req_s"]
    out["rate_serial_sustainable"] = replay(round(sustainable, -2))
    out["rate_serial_sustainable"]["note"] = "0.8 x the one-call-at-a-time throughput measured at 50k req/s"
    out["stats"] = srv.stats()
    srv.close()
    for p in plans:
        p.close()
    return out


# ---------------------------------------------------------- reference arm
def run_reference(args, dist: Dist):
    """The reference's own CPU implementation on the headline workload: rank 0
    alone (other ranks exit without work), every step one parallel run of the
    whole job list on this host's cores.  `value` is the reference's own timed
    form (ntt() per transform); the whole per-call sequence is reported
    beside it.  Nothing here loads libbntt."""
    from benchntt_b200 import workloads as W
    if dist.rank != 0:
        return None
    batch = W.uneven_batch()
    cpu = cpu_uneven(batch.logns, args.steps, args.warmup, max(1, min(args.steps, 10)))
    value = cpu["value"]
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": cpu["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u128 (uint128_t / 2 x u64)",
        "data": "synthetic: seeded uniform residues in [0, q) and seeded per-size twiddle tables",
        "config": workload_config(dist.world),
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def summary(res: dict) -> dict:
    """The figures of the secondary configurations, compact, as the last key
    of the line (rows are lists; "fields" names their entries)."""
    r = lambda v, d=1: None if v is None else round(v, d)
    out = {}
    blas = res.get("blas", {})
    if blas:
        out["blas_2^24"] = {"fields": ["GB/s", "hbm_frac", "e2e_host_GB/s", "cpu_ref_GB/s"]}
        for op, v in blas.items():
            if isinstance(v, dict) and "gbs" in v:
                out["blas_2^24"][op] = [round(v["gbs"]), r(v["frac_of_hbm_peak"], 3),
                                        r(v.get("e2e_host", {}).get("gbs")), r(v.get("cpu_reference_gbs"))]
    pc = res.get("per_call")
    if pc:
        out["per_call"] = {"ntt_per_s": round(pc["value"]), "batched_over_per_call": r(pc["batched_over_per_call"])}
    nl = res.get("new_job_list_each_step")
    if nl:
        out["new_list_vs_same"] = r(nl["vs_same_list"], 3)
    uni = res.get("uniform")
    if uni:
        out["uniform_65536"] = {"fields": ["one_launch_M/s", "per_transform_M/s", "imad80_frac", "cpu_ref_M/s"]}
        for n, v in uni.items():
            m = v["ntt_per_s"] / 1e6
            out["uniform_65536"][n] = [r(m, 1 if m >= 10 else 4), r(v.get("per_transform_ntt_per_s", 0) / 1e6, 3)
                                       if "per_transform_ntt_per_s" in v else None, r(v["imad80_frac"], 3),
                                       r(v.get("cpu_reference_ntt_per_s", 0) / 1e6, 3)
                                       if "cpu_reference_ntt_per_s" in v else None]
    sv = res.get("serving")
    if sv:
        out["serving"] = {"fields": ["rate", "cb_p99_ms", "serial_p99_ms", "p99_speedup", "cb_service_p99_ms",
                                     "serial_service_p99_ms"]}
        for k, v in sv.items():
            if isinstance(v, dict) and "p99_speedup" in v:
                out["serving"][k] = [v["rate_req_s"], r(v["continuous_batching"]["p99_ms"], 3),
                                     r(v["one_call_at_a_time"]["p99_ms"], 3), r(v["p99_speedup"]),
                                     r(v["continuous_batching"]["service_p99_ms"], 3),
                                     r(v["one_call_at_a_time"]["service_p99_ms"], 3)]
    cb = res.get("cpu_baseline")
    if cb:
        out["cpu"] = {"ntt_only": round(cb["value"]), "full_sequence": round(cb["full_sequence"]["value"]),
                      "threads": cb["threads"], "physical_cores": cb["physical_cores"], "smt": cb["smt"],
                      "gpu_over_cpu": r(res["value"] / cb["value"]),
                      "e2e_over_cpu": r(res["e2e"]["value"] / cb["value"], 2) if "e2e" in res else None}
    return out


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
            cpu = cpu_uneven(W.uneven_batch().logns, steps=3, warmup=1, full_steps=2)
            res["cpu_baseline"] = cpu
            res["gpu_over_cpu"] = res["value"] / cpu["value"]
            res["gpu_over_cpu_full_sequence"] = res["value"] / cpu["full_sequence"]["value"]
            res["e2e_over_cpu"] = res["e2e"]["value"] / cpu["value"]
            res["e2e_over_cpu_full_sequence"] = res["e2e"]["value"] / cpu["full_sequence"]["value"]
            ex = cpu_extras(cpu["threads"])
            for n, row in ex["uniform"].items():
                u = res.get("uniform", {}).get(n)
                if u:
                    u["cpu_reference_ntt_per_s"] = row["ntt_per_s"]
                    u["cpu_sample_transforms"] = row["sample_transforms"]
                    u["gpu_over_cpu"] = u["ntt_per_s"] / row["ntt_per_s"]
            one = res.get("single_ntt_1024")
            if one:   # one core per transform, as the reference programs run
                one["cpu_reference_us_per_transform"] = ex["single_ntt_1024_us"]
            for op, row in ex["blas"].items():
                b = res.get("blas", {}).get(op)
                if isinstance(row, dict) and b:
                    b["cpu_reference_gbs"] = row["gbs"]
                    b["gpu_over_cpu"] = b["gbs"] / row["gbs"]
            if "blas" in res:
                res["blas"]["cpu_reference"] = {"impl": ex["blas"]["impl"], "threads": cpu["threads"],
                                                "physical_cores": cpu["physical_cores"], "smt": cpu["smt"]}
        if dist.rank == 0:
            res["summary"] = summary(res)
            print(json.dumps(res), flush=True)
        ctx.close()
    finally:
        dist.close()


if __name__ == "__main__":
    main()

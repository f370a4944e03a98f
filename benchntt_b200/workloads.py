"""Seeded workload definitions for the batched and serving paths.

The reference benchmarks one transform size per process (src/ntt_scalar.c:21,
benchmark/run_ntt.sh:13); the batched engine is measured on mixes of sizes:

  uneven_batch   100,000 transforms with log2 N uniform over 4..10 (N
                 log-uniform over 2^4..2^10), plus 64 at 2^16 and 4 at 2^20,
                 in seeded random order.
  uniform_batch  65,536 transforms of one size.
  serving_trace  Poisson arrivals of mixed NTT / vvmul / axpy requests.

Job buffers are packed back to back in job order; `offsets` gives each job's
first element.  Inputs and per-size twiddle tables are generated from seeds
(bntt_fill_uniform), so every consumer reproduces the same values.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Batch:
    logns: np.ndarray                 # log2 N per job
    offsets: np.ndarray               # first element of each job in the packed buffer
    total: int                        # elements in the packed buffer
    sizes: list = field(default_factory=list)  # distinct log2 N present

    @property
    def count(self) -> int:
        return int(self.logns.shape[0])

    @property
    def butterflies(self) -> int:
        n = 1 << self.logns.astype(np.int64)
        return int(np.sum((n // 2) * self.logns))


def make_batch(logns) -> Batch:
    logns = np.asarray(logns, dtype=np.int64)
    lens = np.left_shift(1, logns)
    offsets = np.zeros(len(logns), dtype=np.int64)
    if len(logns):
        offsets[1:] = np.cumsum(lens)[:-1]
    return Batch(logns=logns, offsets=offsets, total=int(lens.sum()),
                 sizes=sorted(set(int(v) for v in logns)))


def uneven_batch(seed: int = 4, n_small: int = 100_000, small_lo: int = 4, small_hi: int = 10,
                 large=((16, 64), (20, 4))) -> Batch:
    rng = np.random.default_rng(seed)
    small = rng.integers(small_lo, small_hi + 1, size=n_small)
    big = np.concatenate([np.full(c, l) for l, c in large]) if large else np.zeros(0, int)
    logns = np.concatenate([small, big])
    rng.shuffle(logns)
    return make_batch(logns)


def uniform_batch(logn: int, count: int = 65_536) -> Batch:
    return make_batch(np.full(count, logn))


# seeds shared by tests and the benchmark
SEED_INPUT = 11
SEED_TWIDDLE_BASE = 2000    # table for 2^n uses SEED_TWIDDLE_BASE + n


@dataclass
class Request:
    t_arrive: float   # seconds from trace start
    kind: str         # "ntt", "vvmul" or "axpy"
    log2: int         # log2 N (ntt) or log2 length (blas)


def serving_trace(seed: int = 5, rate: float = 50_000.0, count: int = 20_000,
                  ntt_share: float = 0.7, ntt_lo: int = 4, ntt_hi: int = 20,
                  blas_lo: int = 10, blas_hi: int = 22) -> list[Request]:
    """Poisson arrivals at `rate` requests/s: a share `ntt_share` are forward
    NTTs with log2 N uniform over [ntt_lo, ntt_hi], the rest vvmul or axpy
    (equal odds) with log2 length uniform over [blas_lo, blas_hi]."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps) - gaps[0]
    is_ntt = rng.random(count) < ntt_share
    ntt_l = rng.integers(ntt_lo, ntt_hi + 1, size=count)
    blas_l = rng.integers(blas_lo, blas_hi + 1, size=count)
    blas_k = rng.random(count) < 0.5
    out = []
    for i in range(count):
        if is_ntt[i]:
            out.append(Request(float(t[i]), "ntt", int(ntt_l[i])))
        else:
            out.append(Request(float(t[i]), "vvmul" if blas_k[i] else "axpy", int(blas_l[i])))
    return out

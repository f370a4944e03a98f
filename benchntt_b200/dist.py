"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host
side only.

The transforms of a batch are independent, so the data path needs no
collective: each rank runs its own jobs on its own GPU.  The process group
carries barriers around timed regions, the max-over-ranks of a time, and
(for callers that split one job list) nothing else.

Rank, local rank and world size come from the usual launcher variables
(RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


class Dist:
    def __init__(self, backend: str | None = None, timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.pg = dist
            self.backend = backend

    def barrier(self) -> None:
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        """The largest `v` over all ranks (every rank gets it)."""
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def transform_cost(logns) -> np.ndarray:
    """Relative cost of forward transforms: butterflies, N/2 * log2 N."""
    logns = np.asarray(logns, dtype=np.int64)
    return (np.left_shift(1, logns) // 2) * logns


def shard_by_cost(logns, world: int) -> list[np.ndarray]:
    """Splits job indices over `world` ranks, largest transforms first, each
    to the rank with the least work so far (longest-processing-time greedy).
    Every job lands on exactly one rank; the result is the same on every rank
    (deterministic ties), so ranks need not exchange it."""
    cost = transform_cost(logns)
    order = np.lexsort((np.arange(len(cost)), -cost))
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(cost), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += cost[i]
    return [np.nonzero(owner == r)[0] for r in range(world)]

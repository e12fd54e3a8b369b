"""Replicas: one independent run per GPU (the hot path does not shard; the
wakefield step has no exchange between runs).  One process per GPU reads
its rank from the launcher's environment, seeds its run from the rank,
and the job's figures are the maximum time and the summed work over the
ranks, reduced once after the timed region (NCCL on GPUs, gloo on CPUs).
No data-path collective: the runs never exchange particles or fields.
"""
from __future__ import annotations

import datetime
import os

import torch


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def seed(self, base: int) -> int:
        """The run's seed: distinct per rank, the same for every call."""
        return base + 7919 * self.rank

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        if self.backend == "nccl" and torch.cuda.is_available():
            torch.cuda.synchronize()

    def _reduce(self, x: float, op) -> float:
        if not self.dist:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def allmax(self, x: float) -> float:
        """The slowest rank's time: the job's time."""
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def allsum(self, x: float) -> float:
        """The work of all ranks."""
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None

"""Coordination of independent replicas, one process per GPU.

A rounding or RK step is a sequential sweep over the bonds of one train, so
the multi-GPU mode runs N independent trajectories (weak scaling, no
data-path collective).  The process group carries only the barrier around a
timed region and the maximum of the per-rank times (the job's time); the
backend is NCCL on GPUs and gloo on the CPU (tests).
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """rank / world from the launcher's environment (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR, MASTER_PORT); a single process needs no group."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local_rank = int(os.environ.get("LOCAL_RANK", 0))
        self.backend = backend
        self._td = None
        self._torch = None
        if self.world > 1:
            import torch
            import torch.distributed as td

            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            td.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
            self._td, self._torch = td, torch

    def seed(self, base: int) -> int:
        """A different seed per replica (independent trajectories)."""
        return base + self.rank

    def barrier(self) -> None:
        if self._td:
            self._td.barrier()

    def max(self, v: float) -> float:
        """The largest value over the ranks (every rank gets it)."""
        if not self._td:
            return float(v)
        dev = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        t = self._torch.tensor([float(v)], dtype=self._torch.float64, device=dev)
        self._td.all_reduce(t, op=self._td.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj):
        """Every rank's `obj` in rank order (on every rank; a picklable value).
        Used to collect per-instance results (ranks, errors) on rank 0."""
        if not self._td:
            return [obj]
        out = [None] * self.world
        self._td.all_gather_object(out, obj)
        return out

    def job_rate(self, units_per_rank: float, seconds_per_rank: float) -> float:
        """Whole-job throughput: the units all ranks processed over the
        slowest rank's time."""
        return self.world * units_per_rank / self.max(seconds_per_rank)

    def close(self) -> None:
        if self._td:
            self._td.destroy_process_group()
            self._td = None

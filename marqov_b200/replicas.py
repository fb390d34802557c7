"""One independent replica per rank: the multi-GPU plumbing of the engine.

Replicas, temperatures and disorder realisations never exchange data in
MARQOV (one simulation per thread or MPI rank, src/libmarqov/marqovscheduler.h
:64-494), so the data path has no collective: each rank drives its own GPU and
its own replica (replica id = rank).  The only collectives are for timing and
reporting -- a barrier around a timed region and the maximum (or sum) of a
scalar over ranks -- on NCCL for GPU runs and gloo for CPU tests.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


class ReplicaGroup:
    """torchrun-style environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_*);
    a world of one needs no process group."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if self.world > 1 and not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def replica_id(self, base: int = 0) -> int:
        """The replica this rank simulates (24-bit Philox replica field)."""
        return (base + self.rank) & 0xFFFFFF

    def barrier(self):
        if self.world > 1:
            dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return self._reduce(x, dist.ReduceOp.SUM)

    def close(self):
        if self.world > 1 and dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()

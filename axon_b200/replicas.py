"""Replica bookkeeping for runs on several GPUs of one node (one process per GPU).

AXON networks, readout trajectories and recall requests are independent units, so a
multi-GPU run is N replicas: each rank runs its own units on its own GPU, and the only
collectives are a barrier around the timed region and the maximum of the ranks' device
times (the whole job is as slow as its slowest rank). Nothing here moves spikes or weights
between GPUs. torch.distributed is the plumbing: NCCL on GPUs, gloo for the CPU tests.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    """rank / world of this process and the collectives a replica run needs."""

    def __init__(self, rank: int = 0, world: int = 1, dist=None, device: str = "cpu"):
        self.rank, self.world, self.dist, self.device = rank, world, dist, device

    @classmethod
    def from_env(cls, want: int, backend: str = "nccl", timeout_s: float = 120.0) -> "Replicas":
        """Joins the process group that torchrun set up (RANK/WORLD_SIZE/MASTER_* in the
        environment) when more than one replica is wanted; otherwise a single replica."""
        if want <= 1 or "RANK" not in os.environ:
            return cls()
        import torch
        import torch.distributed as dist

        rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
        device = "cpu"
        if backend == "nccl":
            local = int(os.environ.get("LOCAL_RANK", rank))
            torch.cuda.set_device(local)
            device = f"cuda:{local}"
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
        return cls(rank, world, dist, device)

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of x over all ranks (every rank takes this step in the same order)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def shard(self, n: int) -> range:
        """This rank's share of n independent units (contiguous, sizes differ by at most one)."""
        base, extra = divmod(n, self.world)
        lo = self.rank * base + min(self.rank, extra)
        return range(lo, lo + base + (1 if self.rank < extra else 0))

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None

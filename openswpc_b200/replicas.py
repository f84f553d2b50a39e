"""Multi-GPU form of the hot path: independent replicas, no data exchange.

One domain per GPU is the whole time step, so N GPUs run N independent
replicas (or shard the members of an ensemble: 2D models, reciprocity
forces) and meet only to time the job: a barrier before and after the timed
region and the maximum of the per-rank device times.  This module holds that
rank logic; it runs over NCCL on GPUs and over gloo on CPU (the tests).
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    dist: object = None   # torch.distributed when world > 1
    device: str = "cpu"   # tensors for the reductions

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (the job's time is its slowest rank's)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], device=self.device, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def from_env() -> tuple[int, int, int]:
    """(world, rank, local rank) as torchrun sets them."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 600.0) -> Ranks:
    """Joins the process group when torchrun started more than one rank.
    NCCL binds rank r to GPU `local`; gloo reduces on the CPU."""
    world, rank, local = from_env()
    if world <= 1:
        return Ranks(1, 0, local)
    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=timeout_s), device_id=torch.device("cuda", local))
        return Ranks(world, rank, local, dist, f"cuda:{local}")
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return Ranks(world, rank, local, dist, "cpu")


def shard(items, world: int, rank: int) -> list:
    """Members of this rank: every world-th item from `rank` (round robin, so
    uneven members spread over the ranks)."""
    return [x for m, x in enumerate(items) if m % world == rank]


def throughput(units_per_rank: float, steps: int, world: int, ms_max: float) -> float:
    """Whole-job throughput in units per second x 1e-9 (Gcell-updates/s):
    every rank processes `units_per_rank` per step, the job takes the slowest
    rank's time."""
    return units_per_rank * steps * world / (ms_max / 1e3) / 1e9

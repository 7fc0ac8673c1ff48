"""Work distribution over GPUs, one process per GPU.

Gauge configurations are independent, so the multi-GPU form of the path is
replicas: every rank smears and measures its own configurations and no link
data crosses between GPUs. torch.distributed (NCCL on GPUs, gloo on CPU) is
used only for the barrier around timed regions, the max-over-ranks of the
timings and collecting the (small) W tables on rank 0.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def assign(job_sites: Sequence[int], world: int) -> List[List[int]]:
    """Deterministic longest-first assignment of jobs (by site count) to ranks.

    Returns, for each rank, the indices of its jobs in ascending order. Ties
    go to the lower rank, so every rank computes the same assignment.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(job_sites)), key=lambda i: (-int(job_sites[i]), i))
    heap = [(0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(job_sites[i]), r))
    return [sorted(x) for x in out]


def my_jobs(job_sites: Sequence[int], world: int, rank: int) -> List[int]:
    return assign(job_sites, world)[rank]


class Ranks:
    """Thin wrapper over an initialised torch.distributed process group (or a
    single process when there is none)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.rank = self.dist.get_rank() if self.dist else 0
        self.world = self.dist.get_world_size() if self.dist else 1

    def _device(self):
        import torch
        if self.dist and self.dist.get_backend() == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj):
        """Every rank's obj, as a list on rank 0 (None elsewhere)."""
        if not self.dist:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object(obj, out, dst=0)
        return out

"""Multi-GPU plumbing for independent runs ("replicas only").

A single streamer run does not shard: splitting one tree over GPUs would
need a halo exchange after every multigrid half-sweep on every level. What
shards is a set of independent runs (the batched form): runs are assigned
to ranks by estimated cost and each rank steps its own runs with no
data-path collective. The only collectives are the timing reduction (max
over ranks) and optional scalar gathers, done with torch.distributed
(NCCL on GPUs, gloo on CPU in the tests).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a scalar over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(units_all_ranks: float, max_seconds: float) -> float:
    """Whole-job throughput: units processed by all ranks / slowest rank's time."""
    if max_seconds <= 0:
        raise ValueError("time must be positive")
    return units_all_ranks / max_seconds


def partition_runs(costs: Sequence[float], world: int) -> List[List[int]]:
    """Assign independent runs to ranks, longest first onto the least-loaded
    rank (LPT). Deterministic: ties break on rank index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for lst in out:
        lst.sort()
    return out

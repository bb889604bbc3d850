"""Multi-GPU plumbing for independent clouds ("replicas only").

The DSMC step of one cloud exchanges nothing with other clouds, so N GPUs simply run disjoint
sets of clouds: no collective touches the data path.  ``shard_clouds`` balances clouds over
ranks (largest first onto the least-loaded rank); ``aggregate`` combines per-rank timings the
way the benchmark reports them: the job time is the slowest rank, the work is the sum.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def shard_clouds(work: Sequence[float], world_size: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment of clouds (by work, e.g. atoms x steps)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    heap = [(0.0, r) for r in range(world_size)]
    shards: list[list[int]] = [[] for _ in range(world_size)]
    for k in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        load, r = heapq.heappop(heap)
        shards[r].append(k)
        heapq.heappush(heap, (load + float(work[k]), r))
    return [sorted(s) for s in shards]


def aggregate(ms: float, atom_steps: int, group=None) -> tuple[float, int]:
    """(max over ranks of the device time, sum over ranks of atom-steps)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), int(atom_steps)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    a = torch.tensor([float(atom_steps)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(a, op=dist.ReduceOp.SUM, group=group)
    return float(t.item()), int(a.item())

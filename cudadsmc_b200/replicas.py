"""Multi-GPU plumbing for independent clouds ("replicas only").

The DSMC step of one cloud exchanges nothing with other clouds, so N GPUs simply run disjoint
sets of clouds: no collective touches the data path.  ``shard_clouds`` balances clouds over
ranks (largest first onto the least-loaded rank); ``aggregate`` combines per-rank timings the
way the benchmark reports them: the job time is the slowest rank, the work is the sum;
``run_sharded_batch`` runs a batched ensemble split over the ranks (each rank one batched handle
holding its shard) and gathers every cloud's diagnostics on every rank with one small collective
after the run.
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


# per-cloud diagnostics gathered after a sharded run (exact in float64: counts below 2^53, and the
# sums are the handle's own doubles, added to zeros)
GATHERED_FIELDS = ("n_alive", "atom_steps", "collisions", "candidates", "n_evaporated", "n_majorana", "n_knife",
                   "sum_v2", "sum_absB", "e_kin", "e_pot", "e_evaporated", "temperature")


def run_sharded_batch(make_sim, run, clouds, steps: int, seed: int, timer=None, group=None):
    """Runs this rank's shard of `clouds` in one batched handle for `steps` steps.

    make_sim(run, clouds) builds the handle (the engine's Simulation, or anything with its
    interface); timer(fn) runs fn and returns its device time in ms (default: wall clock).  Every
    rank calls this with the same arguments.  Returns (ms over ranks' max, atom-steps summed over
    ranks, table): table[k] is cloud k's diagnostics (GATHERED_FIELDS), whichever rank ran it,
    gathered by one all-reduce of a (clouds x fields) float64 tensor in which every rank fills only
    its own rows."""
    import time
    import numpy as np
    import torch
    import torch.distributed as dist
    dist_on = dist.is_available() and dist.is_initialized()
    ws = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    shard = shard_clouds([float(c.n_atoms) for c in clouds], ws)[rank]
    rows = np.zeros((len(clouds), len(GATHERED_FIELDS)), np.float64)
    ms = 0.0
    atom_steps = 0
    if shard:
        sim = make_sim(run, [clouds[k] for k in shard])
        sim.init_cloud(seed)
        d0 = sim.diagnostics()

        def work():
            sim.step(steps)
            sim.synchronize()

        if timer is None:
            t0 = time.perf_counter()
            work()
            ms = (time.perf_counter() - t0) * 1e3
        else:
            ms = timer(work)
        atom_steps = sim.diagnostics()["atom_steps"] - d0["atom_steps"]
        for j, k in enumerate(shard):
            d = sim.diagnostics(j)
            rows[k] = [float(d[f]) for f in GATHERED_FIELDS]
        sim.close()
    if dist_on:
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(rows).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        rows = t.cpu().numpy()
    ms, atom_steps = aggregate(ms, atom_steps, group)
    table = [dict(zip(GATHERED_FIELDS, r)) for r in rows]
    return ms, atom_steps, table

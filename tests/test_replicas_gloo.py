"""Replicas on CPU with world size 2 (gloo): clouds sharded over ranks evolve exactly as in one
process, and the throughput aggregation takes the slowest rank and sums the work.  The sharded
batched run (replicas.run_sharded_batch, the path of `bench.py --batched` under torchrun) is run
with the oracle standing in for the engine's Python layer (it has the same interface), and every
cloud's gathered diagnostics must equal a one-process run of the whole batch."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cudadsmc_b200.replicas import shard_clouds


def clouds(k=5):
    import oracle
    out = []
    rng = np.random.default_rng(5)
    for i in range(k):
        run, c = oracle.preset(2)
        c.n_atoms = c.capacity = int(rng.integers(300, 3000))
        c.cells[0] = c.cells[1] = c.cells[2] = 10
        c.alpha = 3000.0
        c.stream_id = 40 + i
        out.append(c)
    return run, out


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import oracle
    from cudadsmc_b200.replicas import aggregate
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    run, cl = clouds()
    shard = shard_clouds([c.n_atoms for c in cl], world)[rank]
    o = oracle.Oracle(run, [cl[k] for k in shard])
    o.init_cloud(1234)
    o.step(6)
    mine = {k: o.diagnostics(j) for j, k in enumerate(shard)}
    ms, steps = aggregate(10.0 * (rank + 1), mine and sum(d["atom_steps"] for d in mine.values()) or 0)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        q.put((ms, steps, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_balance():
    shards = shard_clouds([10, 9, 8, 1, 1, 1], 2)
    assert sorted(sum(shards, [])) == list(range(6))
    loads = sorted(sum([10, 9, 8, 1, 1, 1][k] for k in s) for s in shards)
    assert loads == [13, 17]  # the best split of these sizes
    assert sorted(sum(shard_clouds([5, 5, 5, 5], 4), [])) == [0, 1, 2, 3]


def test_two_rank_replicas_match_single_process():
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ms, steps, gathered = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert ms == 20.0
    run, cl = clouds()
    ref = oracle.Oracle(run, cl)
    ref.init_cloud(1234)
    ref.step(6)
    merged = {}
    for part in gathered:
        merged.update(part)
    assert sorted(merged) == list(range(len(cl)))
    total = 0
    for k, d in merged.items():
        r = ref.diagnostics(k)
        for f in ("n_alive", "sum_v2", "sum_absB", "collisions", "n_evaporated", "atom_steps"):
            assert d[f] == r[f], (k, f)
        total += d["atom_steps"]
    assert steps == total


def _sharded_worker(rank, world, port, q):
    import torch.distributed as dist
    import oracle
    from cudadsmc_b200.replicas import run_sharded_batch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    run, cl = clouds(7)
    ms, steps, table = run_sharded_batch(lambda r, c: oracle.Oracle(r, c), run, cl, steps=5, seed=77,
                                         timer=lambda fn: (fn(), 3.0 * (rank + 1))[1])
    q.put((rank, ms, steps, table))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_gathers_every_cloud():
    import oracle
    from cudadsmc_b200.replicas import GATHERED_FIELDS, run_sharded_batch
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    run, cl = clouds(7)
    ms1, steps1, ref = run_sharded_batch(lambda r, c: oracle.Oracle(r, c), run, cl, steps=5, seed=77)
    for rank, ms, steps, table in got:
        assert ms == 6.0  # the slowest rank
        assert steps == steps1
        for k in range(len(cl)):
            for f in GATHERED_FIELDS:
                assert table[k][f] == ref[k][f], (rank, k, f)

"""Multi-rank host logic on CPU (gloo, world_size 2): energy sharding and the
max-over-ranks timing reduction the benchmark uses.  No GPU involved."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from scatt_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_covers_every_energy_once():
    rng = np.random.default_rng(1)
    for n, world in [(200, 1), (200, 2), (256, 8), (7, 4), (3, 8)]:
        lc = rng.choice([12, 16, 20], size=n)
        parts = shard.partition(shard.energy_cost(lc, 605), world)
        assert len(parts) == world
        allidx = np.concatenate(parts)
        assert np.array_equal(np.sort(allidx), np.arange(n))
        for p in parts:
            assert p.size == 0 or np.array_equal(p, np.arange(p[0], p[-1] + 1))


def test_partition_balances_cost():
    lc = np.array([20] * 100 + [12] * 100)
    costs = shard.energy_cost(lc, 605)
    parts = shard.partition(costs, 2)
    c = [costs[p].sum() for p in parts]
    assert abs(c[0] - c[1]) / sum(c) < 0.02


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ks = np.linspace(0.05, 2.0, 50)
    lc = np.where(np.arange(50) % 3 == 0, 20, 12)
    parts = shard.partition(shard.energy_cost(lc, 605), world)
    mine = parts[rank]
    # each rank "solves" its block: deterministic per-energy payload
    payload = torch.tensor([float(i) for i in mine], dtype=torch.float64)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([payload.numel()]))
    maxn = int(max(s.item() for s in sizes))
    padded = torch.full((maxn,), -1.0, dtype=torch.float64)
    padded[: payload.numel()] = payload
    gathered = [torch.zeros(maxn, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(gathered, padded)
    # max-over-ranks timing, as in bench.py
    t = torch.tensor([1.0 + rank, 10.0 * (rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        got = sorted(int(x) for g in gathered for x in g.tolist() if x >= 0)
        q.put((got, t.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_and_max_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == list(range(50))
    assert t == [2.0, 20.0]

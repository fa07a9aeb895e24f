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


def _tau_worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    k, D = _smooth_dipoles(sum(sizes))
    lo = sum(sizes[:rank])
    mine = slice(lo, lo + sizes[rank])
    tau = shard.halo_time_delay(k[mine], D[mine])
    q.put((rank, tau.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def _smooth_dipoles(n):
    """An uneven k grid and smooth complex dipoles of 5 channels on it."""
    k = np.sort(np.random.default_rng(7).uniform(0.05, 2.0, n))
    ch = np.arange(5)[None, :]
    D = (1.0 + 0.3 * ch) * np.exp(1j * (0.8 * k[:, None] + 0.2 * ch * k[:, None] ** 2)) / (1.0 + k[:, None])
    return k, D


@pytest.mark.parametrize("sizes", [(13, 17), (9, 0, 11), (1, 1, 12)])
def test_time_delay_with_k_halo_equals_whole_grid(sizes):
    """Ranks holding contiguous blocks of the k grid (some of one energy, one
    empty) get, with the one-point halo, the whole grid's delay at every
    energy: the finite difference at a block edge uses the neighbour's edge
    energy."""
    from scatt_b200.observables import time_delay
    world = len(sizes)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_tau_worker, args=(r, world, port, list(sizes), q)) for r in range(world)]
    for p in procs:
        p.start()
    parts = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = np.concatenate([np.array(parts[r]) for r in range(world)])
    k, D = _smooth_dipoles(sum(sizes))
    ref = time_delay(k, D)
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))
    # without the halo the block edges differ (one-sided differences there)
    own = np.concatenate([time_delay(k[a:a + s], D[a:a + s]) for a, s in
                          zip(np.cumsum((0,) + sizes[:-1]), sizes) if s >= 2])
    if sizes == (13, 17):
        assert np.max(np.abs(own - ref)) > 1e-6 * np.max(np.abs(ref))

"""Energy sharding across ranks (one process per GPU).

Energies are independent (src/main.cpp:847-877; the reference's own launcher
block-splits [ik_min, ik_max] over MPI ranks, src/run_mpi.cpp:9-11).  Each
rank gets one contiguous block of the k grid; with mixed continuum cutoffs
the blocks are balanced by the per-energy cost, dominated by the N_t^3
inversions of the R-ratio recurrence.  No collective runs on the solve's
data path; ranks agree on the partition, reduce a max for timing, and, for
the time delay (a finite difference across energies), exchange their edge
energies with their neighbours once the scan is done (halo_time_delay).
"""
from __future__ import annotations

import numpy as np


def energy_cost(l_cont: np.ndarray, n_f: int) -> np.ndarray:
    """Relative cost of one energy: N_t^3 with N_t = (l_cont + 1)^2 + N_f."""
    nt = (np.asarray(l_cont, dtype=np.float64) + 1.0) ** 2 + n_f
    return nt ** 3


def partition(costs, world: int) -> list[np.ndarray]:
    """Contiguous blocks, one per rank, with near-equal summed cost.

    Greedy cut of the cost prefix sum at multiples of total / world; every
    index appears in exactly one block and blocks keep the k-grid order.
    """
    costs = np.asarray(costs, dtype=np.float64)
    n = costs.size
    if world <= 1 or n == 0:
        return [np.arange(n)]
    csum = np.cumsum(costs)
    total = csum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        c = int(np.searchsorted(csum, target, side="left")) + 1
        c = min(max(c, cuts[-1]), n)
        cuts.append(c)
    cuts.append(n)
    return [np.arange(cuts[r], cuts[r + 1]) for r in range(world)]


def halo_time_delay(k_block, D_block, with_minus: bool = False, group=None) -> np.ndarray:
    """Wigner delay over this rank's contiguous block of the k grid, equal at
    every point of the block to observables.time_delay over the whole grid.

    tau needs dD/dk by finite differences across energies, so at a block
    edge it needs the neighbouring rank's edge energy: a one-point k-halo.
    One all_gather of every rank's first and last (k, D) rows supplies it;
    an edge with no neighbour (the ends of the grid) keeps the one-sided
    difference the whole-grid computation uses there.  Collective: every
    rank of the group calls it, with D_block of shape (n, n_channels) even
    when its block is empty (n = 0)."""
    import torch
    import torch.distributed as dist

    from .observables import time_delay
    k_block = np.asarray(k_block, dtype=np.float64).reshape(-1)
    D_block = np.asarray(D_block, dtype=np.complex128)
    n, n_ch = D_block.shape
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    edge = torch.zeros(2, 2 + 2 * n_ch, dtype=torch.float64)    # [present, k, Re D, Im D]
    if n:
        for j, i in enumerate((0, n - 1)):
            edge[j, 0] = 1.0
            edge[j, 1] = k_block[i]
            edge[j, 2:2 + n_ch] = torch.from_numpy(D_block[i].real.copy())
            edge[j, 2 + n_ch:] = torch.from_numpy(D_block[i].imag.copy())
    edge = edge.to(dev)
    got = [torch.zeros_like(edge) for _ in range(world)]
    dist.all_gather(got, edge, group=group)
    got = [g.cpu().numpy() for g in got]
    if not n:
        return np.zeros(0)
    row = lambda r: (r[1], r[2:2 + n_ch] + 1j * r[2 + n_ch:])
    left = next((row(g[1]) for g in reversed(got[:rank]) if g[0, 0] > 0), None)
    right = next((row(g[0]) for g in got[rank + 1:] if g[0, 0] > 0), None)
    ks, Ds, lo = [k_block], [D_block], 0
    if left is not None:
        ks.insert(0, [left[0]])
        Ds.insert(0, left[1][None])
        lo = 1
    if right is not None:
        ks.append([right[0]])
        Ds.append(right[1][None])
    tau = time_delay(np.concatenate(ks), np.concatenate(Ds), with_minus)
    return tau[lo:lo + n]

"""Energy sharding across ranks (one process per GPU).

Energies are independent (src/main.cpp:847-877; the reference's own launcher
block-splits [ik_min, ik_max] over MPI ranks, src/run_mpi.cpp:9-11).  Each
rank gets one contiguous block of the k grid; with mixed continuum cutoffs
the blocks are balanced by the per-energy cost, dominated by the N_t^3
inversions of the R-ratio recurrence.  No collective runs on the data path;
ranks only agree on the partition and, for timing, reduce a max.
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

"""Gauss-Jordan inverse with tournament pivoting.  TEST INFRASTRUCTURE ONLY.

The device inverse picks one pivot per column with a block-wide argmax
and barrier (partial pivoting, as LAPACK's dgetrf).  The planned change
picks a whole 16-column panel's pivots at once: each block of rows
proposes candidates by partial-pivot LU on its own rows, and one more LU
over the candidates picks the winners (tournament pivoting, as in
communication-avoiding LU).  That changes the pivot sequence, so results
change at the rounding level.  This module states the scheme on the CPU;
the tests run the oracle's whole solve with it and hold the change to
the spread the oracle's two LAPACK builds already show.
"""
from __future__ import annotations

import numpy as np


def _lu_pick(P: np.ndarray, b: int) -> np.ndarray:
    """Row indices (into P) that partial-pivot LU of the m x b panel P picks, in order."""
    P = P.copy()
    m = P.shape[0]
    idx = np.arange(m)
    for j in range(min(b, m)):
        p = j + int(np.argmax(np.abs(P[j:, j])))
        P[[j, p]] = P[[p, j]]
        idx[[j, p]] = idx[[p, j]]
        if P[j, j] != 0.0:
            P[j + 1:, j:] -= np.outer(P[j + 1:, j] / P[j, j], P[j, j:])
    return idx[: min(b, m)]


def gj_inverse_tournament(A: np.ndarray, panel: int = 16, blocks: int = 4) -> np.ndarray:
    """A^-1 by Gauss-Jordan on [A | I]; the pivots of each `panel` columns
    come from a tournament over `blocks` row blocks of the remaining rows."""
    n = A.shape[0]
    M = np.hstack([np.asarray(A, dtype=np.float64), np.eye(n)])
    done = 0
    while done < n:
        bw = min(panel, n - done)
        rows = np.arange(done, n)
        cand = []
        for blk in np.array_split(rows, min(blocks, rows.size)):
            cand.extend(blk[_lu_pick(M[blk, done:done + bw], bw)])
        cand = np.asarray(cand)
        winners = cand[_lu_pick(M[cand, done:done + bw], bw)]
        # bring the winners, in order, to rows done .. done + bw - 1
        where = np.arange(n)                   # current row of each original row
        at = np.arange(n)                      # original row now at each row
        for j, w in enumerate(winners):
            tgt, cur = done + j, where[w]
            if tgt != cur:
                M[[tgt, cur]] = M[[cur, tgt]]
                a_t, a_c = at[tgt], at[cur]
                at[tgt], at[cur] = a_c, a_t
                where[a_c], where[a_t] = tgt, cur
        for j in range(bw):
            c = done + j
            if M[c, c] == 0.0:
                raise np.linalg.LinAlgError("gj_inverse_tournament: zero pivot")
            M[c] /= M[c, c]
            f = M[:, c].copy()
            f[c] = 0.0
            M -= np.outer(f, M[c])
        done += bw
    return M[:, n:]

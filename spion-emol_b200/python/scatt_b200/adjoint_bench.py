"""Timing of the device adjoint on the adjoint workload's shape.

    python -m scatt_b200.adjoint_bench [--energies 16] [--segment 256] [--Nr 12001] [--dr 0.005]

Workload: the H2O-like system at l_cont = 12 (169 continuum + 605 exchange
channels, N_t = 774), 12001 radial points at dr = 0.005, momenta spread over
0.05 .. 2.0, seeded synthetic inputs of those shapes.  One pass is the
forward sweep with R-ratio checkpoints every `segment` points
(scatt_adjoint_forward), the dipoles and a scalar objective on them in torch,
its backward pass, and the library's reverse sweep with segment recompute
(scatt_adjoint_reverse) giving tr dJ/dV(n) for every energy and dJ/dV(n)
summed over the energies.  Prints one JSON line with the seconds of each
part (host clock around device-synchronised calls) and energies/s.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import adjoint as ADJ
from . import solver as S
from . import synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--energies", type=int, default=16)
    ap.add_argument("--segment", type=int, default=256)
    ap.add_argument("--Nr", type=int, default=12001)
    ap.add_argument("--dr", type=float, default=0.005)
    ap.add_argument("--l-cont", type=int, default=12)
    ap.add_argument("--reps", type=int, default=1)
    a = ap.parse_args(argv)
    inp = synth.h2o_like(Nr=a.Nr, dr=a.dr, l_cont=a.l_cont, lmax_orb=40, n_orb=5)
    sol = S.ScanSolver(inp)
    ks = np.linspace(0.05, 2.0, a.energies)
    Es = 0.5 * ks ** 2
    rng = np.random.default_rng(3)
    weights = [torch.as_tensor(rng.standard_normal(sol.Np), device="cuda") for _ in range(6)]

    def one_pass():
        t0 = time.time()
        adj = ADJ.ScanAdjoint(sol, Es, segment=a.segment)
        torch.cuda.synchronize()
        t1 = time.time()
        J = 0.0
        for Ds in adj.dipoles():
            for s in range(6):
                J = J + torch.sum(weights[s] * torch.abs(Ds[s]) ** 2)
        J.backward()
        torch.cuda.synchronize()
        t2 = time.time()
        vtr, vfull = adj.reverse(full=True)
        torch.cuda.synchronize()
        t3 = time.time()
        ok = bool(np.all(np.isfinite(vtr))) and bool(torch.isfinite(vfull).all())
        adj.close()
        return t1 - t0, t2 - t1, t3 - t2, ok

    runs = [one_pass() for _ in range(a.reps)]
    fwd, mid, rev, ok = runs[-1]
    total = fwd + mid + rev
    print(json.dumps({
        "workload": "h2o_like adjoint", "Nr": a.Nr, "dr": a.dr, "l_cont": a.l_cont, "N_t": sol.Np + sol.Nf,
        "energies": a.energies, "segment": a.segment,
        "forward_s": fwd, "torch_stages_s": mid, "reverse_s": rev, "total_s": total,
        "energies_per_s": a.energies / total, "finite": ok,
    }))


if __name__ == "__main__":
    main()

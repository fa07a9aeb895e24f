"""Timing of the psi store and its continuum-continuum consumer.

    python -m scatt_b200.psi_bench [--nr 801] [--energies 4] [--points 400] [--segment 64] [--nu 3]

On the H2O-like channel set (l_cont 20: N_psi 441, N_t 1046) over a short
radial grid: one batch through scatt_solve_batch (fit accumulated forward),
then the same energies through scatt_psi_sweep writing psi(n) for the last
`points` points below n_transition into page-locked host memory, then
scatt_cc_dipole of the first energy against the next `nu`.  Host clock
around each call (every call synchronises before it returns).  Prints one
JSON line: seconds of each call, the sweep's overhead over the plain solve,
the bytes of psi streamed to the host and their rate, and the cc
contraction's FP64 rate (2 N_psi^3 flops per point and pair) with the bytes
of psi_nu it copies to the device.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib, synth
from . import solver as S


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nr", type=int, default=801)
    ap.add_argument("--energies", type=int, default=4)
    ap.add_argument("--points", type=int, default=400)
    ap.add_argument("--segment", type=int, default=64)
    ap.add_argument("--nu", type=int, default=3)
    a = ap.parse_args(argv)
    import torch
    inp = synth.h2o_like(Nr=a.nr, dr=0.005, l_cont=20, lmax_orb=40, n_orb=5)
    sol = S.ScanSolver(inp, device=0)
    Es = 0.5 * np.linspace(0.6, 1.6, a.energies) ** 2
    o = S.default_opts(allow_closed_channels=1, keep_window=0)
    sol.solve(Es[:1], opts=o)                      # warm-up: module load, tables
    t0 = time.perf_counter()
    sol.solve(Es, opts=o)
    t_solve = time.perf_counter() - t0
    n_hi = min(inp.Nr, sol.n_transition)
    n_lo = max(0, n_hi - a.points)
    keep = []

    def pinned(shape, dtype=np.float64):
        t = torch.zeros(shape, dtype=torch.float64, pin_memory=True)
        keep.append(t)
        return t.numpy()

    t0 = time.perf_counter()
    _, psi = sol.psi_sweep(Es, n_lo=n_lo, n_hi=n_hi, segment=a.segment, opts=o, alloc=pinned)
    t_sweep = time.perf_counter() - t0
    psi_bytes = int(keep[0].numel() * 8)
    nu = min(a.nu, a.energies - 1)
    pk, pn = psi[0], psi[1:1 + nu]                  # views of the page-locked buffer, no copies
    _lib.cc_dipole(pk[:8], pn[:, :8], n_lo, inp.dr, "z")     # warm-up
    t0 = time.perf_counter()
    _lib.cc_dipole(pk, pn, n_lo, inp.dr, "z")
    t_cc = time.perf_counter() - t0
    Np = sol.Np
    flops = 2.0 * Np ** 3 * (n_hi - n_lo) * nu
    print(json.dumps({
        "workload": f"h2o_like l_cont 20 (N_psi {Np}, N_t {Np + sol.Nf}), Nr {inp.Nr}, n_transition "
                    f"{sol.n_transition}, {a.energies} energies, psi over [{n_lo}, {n_hi}), segment {a.segment}",
        "solve_s": t_solve, "psi_sweep_s": t_sweep, "sweep_over_solve": t_sweep / t_solve,
        "psi_bytes_to_host": psi_bytes, "psi_GBps_to_host": psi_bytes / t_sweep / 1e9,
        "cc_pairs": nu, "cc_points": n_hi - n_lo, "cc_s": t_cc, "cc_tflops": flops / t_cc / 1e12,
        "cc_bytes_to_device": int((nu + 1) * (n_hi - n_lo) * Np * Np * 8)}))
    sol.close()


if __name__ == "__main__":
    main()

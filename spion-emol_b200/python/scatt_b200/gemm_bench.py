"""Device timing of the batched FP64 GEMMs of the scan's Schur and W^-1 stages.

    python -m scatt_b200.gemm_bench [--np 441] [--nf 605] [--slots 128] [--reps 5]

The products of one chunk of the H2O-like scan (Np = 441 continuum and
N_f = 605 exchange channels): the Schur update S -= Bs B^T (Np x Np x N_f,
symmetric, one per slot and radial step of the chunk: 8 x slots), T = Sinv Bs
(Np x N_f x Np) and F = Bs^T T (N_f x N_f x Np, symmetric), one per slot.
CUDA events bracket the batched call only (scatt_bench_gemm).  Prints one
JSON line per product with ms per call and the FP64 rate: 2 M N K per
product, counted as M (M + 1) K for the symmetric ones (the lower triangle
and the diagonal), against the cuBLAS DGEMM 8192^3 rate measured in the same
process (torch.matmul).
"""
from __future__ import annotations

import argparse
import json

from . import _lib


def dgemm_peak():
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = 1e30
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 2.0 * n ** 3 / best / 1e12


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--np", type=int, default=441)
    ap.add_argument("--nf", type=int, default=605)
    ap.add_argument("--slots", type=int, default=128)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    peak = dgemm_peak()
    Np, Nf, S = a.np, a.nf, a.slots
    cases = [("schur_update_S", 0, 1, Np, Np, Nf, 8 * S, True),
             ("T_sinv_bs", 0, 0, Np, Nf, Np, S, False),
             ("F_bst_t", 1, 0, Nf, Nf, Np, S, True)]
    for name, oa, ob, M, N, K, cnt, sym in cases:
        ms = _lib.bench_gemm(oa, ob, M, N, K, cnt, sym, a.reps)
        flops = (M * (M + 1) * K if sym else 2 * M * N * K) * cnt
        tf = flops / (ms * 1e-3) / 1e12
        print(json.dumps({"product": name, "opA": oa, "opB": ob, "M": M, "N": N, "K": K, "count": cnt, "sym": sym,
                          "ms_per_call": ms, "tflops": tf, "dgemm_tflops": peak, "frac_of_dgemm": tf / peak}))


if __name__ == "__main__":
    main()

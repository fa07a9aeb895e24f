"""Device timing of the batched FP64 inverse (the per-step R^-1 / Sinv kernels).

    python -m scatt_b200.inverse_bench --n 1046 --count 32 [--reps 5] [--scheme 0|1|2|3|4]

Seeded well-conditioned matrices are generated on the device; CUDA events
bracket the inverse kernels only (scatt_bench_inverse).  Prints one JSON line
per order with ms per call and the achieved FP64 rate counted as 2 n^3 flops
per matrix.
"""
from __future__ import annotations

import argparse
import json

from . import _lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, nargs="+", default=[1046])
    ap.add_argument("--count", type=int, default=32)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--scheme", type=int, default=0,
                    help="0 automatic (default), 1 single-level, 2 two-level column-major, "
                         "3 two-level row-contiguous, 4 as 3 with 128-column windows")
    a = ap.parse_args(argv)
    _lib.set_inverse_blocking(a.scheme)
    for n in a.n:
        ms = _lib.bench_inverse(n, a.count, a.reps)
        print(json.dumps({"n": n, "count": a.count, "reps": a.reps,
                          "scheme": a.scheme,
                          "ms_per_call": ms, "tflops": 2.0 * n ** 3 * a.count / (ms * 1e-3) / 1e12}))


if __name__ == "__main__":
    main()

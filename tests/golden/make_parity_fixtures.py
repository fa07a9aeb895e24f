"""Oracle fixtures for GPU parity at the benchmark shapes.

    python tests/golden/make_parity_fixtures.py CASE [--threads T] [--accum]

CASE is one of:
  h2_c1        the H2-like workload at its full size (Nr 4001, dr 0.01,
               l_cont 8): k = 0.1, 1.0, 2.0;
  h2o_nt1046   the H2O-like channel set at l_cont 20 (N_t = 1046, so the
               solver's R^-1 runs the row-contiguous look-ahead inverse) on a
               short grid (Nr 601, dr 0.05): k = 0.6, 1.5;
  h2o_c2       the H2O-like workload at its full size (Nr 12001, dr 0.005,
               l_cont 20): k = 1.0, 0.05.

Each energy is solved by the oracle in both LAPACK builds (Eigen partial-pivot
LU and MKL dgetri / dsytrf + dsytri); their spread is the rounding floor the
GPU tests scale their tolerance by.  Matrices with more than 100 rows are
stored as products with four seeded random vectors plus their diagonals,
which checks every entry with probability one at a fraction of the size.
With --accum the six dipoles are also computed by the oracle's restatement
of the GPU's own order of summation (oracle/adjoint_recurrence.DipoleAdjoint:
the dipole rows accumulated forward with the R-ratios, Q = G(N-1)^T Z_N,
instead of a back sweep), stored as e<i>/accum/{D, D_raw, d_raw}: the spread between the
two summation orders is the floor of the dipoles where they are
ill-conditioned.
The file is tests/golden/parity_CASE.npz; it is rewritten after every solve,
so a long case keeps what it has finished.  The full-size grids use the
oracle's checkpointed solve (solve_energy_lean), whose results equal
solve_energy's bit for bit.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

CASES = {
    "h2_c1": dict(builder="h2_like", kw=dict(Nr=4001, dr=0.01, l_cont=8), ks=[0.1, 1.0, 2.0]),
    "h2o_nt1046": dict(builder="h2o_like", kw=dict(Nr=601, dr=0.05, l_cont=20, lmax_orb=40, n_orb=5),
                       ks=[0.6, 1.5]),
    "h2o_c2": dict(builder="h2o_like", kw=dict(Nr=12001, dr=0.005, l_cont=20, lmax_orb=40, n_orb=5),
                   ks=[1.0, 0.05]),
}
FULL_LIMIT = 100      # matrices up to this order are stored whole
PROJ_SEED = 7


def proj_vectors(Np):
    import numpy as np
    return np.random.default_rng(PROJ_SEED).standard_normal((Np, 4))


def reduce_matrix(M, V):
    import numpy as np
    M = np.asarray(M)
    if M.shape[0] <= FULL_LIMIT:
        return {"full": M}
    return {"proj": M @ V, "diag": np.diag(M).copy()}


def record(r, V):
    """The fields of one oracle result the GPU tests compare."""
    import numpy as np
    out = {}
    for name, M in (("K_kme", r.K_kme), ("A", r.aa["A"]), ("B", r.aa["B"]), ("K_aa", r.aa["K"])):
        for k, v in reduce_matrix(M, V).items():
            out[f"{name}.{k}"] = v
    out["b_overlap"] = np.asarray(r.b_overlap)
    for key in ("D", "D_raw", "d_raw", "d_corr", "partial_sigma"):
        out[key] = np.array([np.asarray(r.slices[s][key]) for s in range(6)])
    out["eig_kme"] = np.sort(np.asarray(r.kme["eigenphases"]))
    out["shifts"] = np.array([r.shifts["A"], r.shifts["S"]])
    out["fit"] = np.array([r.aa["n_fit_start"], r.aa["n_fit_end"], r.aa["fit_residual_rel"]])
    out["n_closed_l"] = np.array(len(r.aa["closed_l"]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=list(CASES))
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--accum", action="store_true")
    a = ap.parse_args()
    if a.threads:
        for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
            os.environ[v] = str(a.threads)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "spion-emol_b200", "python"))
    import numpy as np

    from oracle import solver as O
    from scatt_b200 import synth

    cfg = CASES[a.case]
    inp = getattr(synth, cfg["builder"])(**cfg["kw"])
    st = O.make_setup(inp)
    V = proj_vectors(st.n_mu)
    path = os.path.join(HERE, f"parity_{a.case}.npz")
    data = {"ks": np.array(cfg["ks"]), "proj_vectors": V, "n_tr": np.array(st.n_tr),
            "Nt": np.array(st.Nt), "Np": np.array(st.n_mu)}
    if os.path.exists(path):
        old = dict(np.load(path))
        data.update({k: v for k, v in old.items() if "/" in k})
    lean = st.Nr > 2000
    for ik, k in enumerate(cfg["ks"]):
        E = 0.5 * k * k
        for build in ("eigen", "mkl"):
            tag = f"e{ik}/{build}/"
            if any(key.startswith(tag) for key in data):
                continue
            O.BUILD = build
            t0 = time.time()
            r = O.solve_energy_lean(st, E) if lean else O.solve_energy(st, E)
            for key, v in record(r, V).items():
                data[tag + key] = v
            np.savez_compressed(path, **data)
            print(f"{a.case} k={k} {build}: {time.time() - t0:.0f} s", flush=True)
    if a.accum:
        from oracle import adjoint_recurrence as AR
        O.BUILD = "eigen"
        for ik, k in enumerate(cfg["ks"]):
            if f"e{ik}/accum/D_raw" in data:
                continue
            t0 = time.time()
            da = AR.DipoleAdjoint(st, 0.5 * k * k, lambda n: O.V_at(st, n))
            data[f"e{ik}/accum/D"] = np.array(da.dipoles())
            # D_raw = ((A - iB)^-1)^dagger d_raw, d_raw = the first six rows of Q
            M = np.linalg.inv(da.A.astype(complex) - 1j * da.B).conj().T
            data[f"e{ik}/accum/D_raw"] = (M @ da.Q[:6].T).T
            data[f"e{ik}/accum/d_raw"] = np.array(da.Q[:6])
            np.savez_compressed(path, **data)
            print(f"{a.case} k={k} accum: {time.time() - t0:.0f} s", flush=True)
    O.BUILD = "eigen"


if __name__ == "__main__":
    main()

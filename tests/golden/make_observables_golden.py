"""Golden vectors of the reference's own observables code
(postprocessing/cross_section_delay.py), run on seeded dipoles.

The reference module is imported from REF (the required first argument) and
its numerical functions run unmodified: sigma_from_dipole, time_delay (both
sign conventions), q_sigma, dphi_rms and compute_beta.  Only its plotting
uses matplotlib, which this image lacks, so a stand-in module with use()
and pyplot is put into sys.modules before the import.

    python tests/golden/make_observables_golden.py REF
"""
import json
import os
import sys
import types

import numpy as np

if len(sys.argv) < 2:
    sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, os.path.join(REF, "postprocessing"))
    import cross_section_delay
    return cross_section_delay


def main():
    R = load_reference()
    rng = np.random.default_rng(20261204)
    n_e, l_max = 6, 3
    n_ch = (l_max + 1) ** 2
    k = np.sort(rng.uniform(0.3, 1.8, n_e))
    omega = 0.5 * k ** 2 + 0.46
    D = [rng.standard_normal((n_e, n_ch)) + 1j * rng.standard_normal((n_e, n_ch)) for _ in range(6)]
    slots = [("length", "x"), ("length", "y"), ("length", "z"),
             ("velocity", "x"), ("velocity", "y"), ("velocity", "z")]
    out = {"k": k.tolist(), "omega": omega.tolist(),
           "D_re": [d.real.tolist() for d in D], "D_im": [d.imag.tolist() for d in D]}
    for s, (g, p) in enumerate(slots):
        out[f"sigma_{g}_{p}"] = R.sigma_from_dipole(k, D[s], omega, g).tolist()
        out[f"tau_{g}_{p}"] = R.time_delay(k, D[s]).tolist()
        out[f"tau_minus_{g}_{p}"] = R.time_delay(k, D[s], with_minus=True).tolist()
    for p, pol in enumerate("xyz"):
        out[f"q_{pol}"] = R.q_sigma(D[p], D[3 + p], omega).tolist()
        out[f"dphi_rms_{pol}"] = R.dphi_rms(D[p], D[3 + p]).tolist()
    for g, gauge in enumerate(("length", "velocity")):
        out[f"beta_{gauge}"] = R.compute_beta(D[3 * g], D[3 * g + 1], D[3 * g + 2], list(range(n_ch))).tolist()
    with open(os.path.join(HERE, "observables_vectors.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()

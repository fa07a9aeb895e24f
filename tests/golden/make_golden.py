"""Extract the golden vectors of the reference's own unit tests into JSON.

Reads (text only, nothing is compiled or run):
  src/tests/test_real_gaunt_dipole.cpp   kGoldStandard real-Y Gaunt table (l <= 3, q = -1, 0, +1)
  src/tests/test_gaunt.cpp               permutation-symmetry cases
  src/tests/test_freeparticle_dipole.cpp free-particle k list, grid and tolerances

Run with the path of a reference checkout as REF (required):
    python tests/golden/make_golden.py REF
"""
import json
import os
import re
import sys

if len(sys.argv) < 2:
    sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
REF = sys.argv[1]
HERE = os.path.dirname(os.path.abspath(__file__))


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def main():
    out = {}
    src = read("src/tests/test_real_gaunt_dipole.cpp")
    body = src[src.index("kGoldStandard"):]
    body = body[: body.index("};")]
    rows = re.findall(r"\{\s*(-?\d+),\s*(-?\d+),\s*([+-]?\d+),\s*(-?\d+),\s*(-?\d+),\s*([+-]?[0-9.]+)\s*\}", body)
    out["real_gaunt_dipole"] = [
        {"l_mu": int(a), "m_mu": int(b), "q": int(c), "l_nu": int(d), "m_nu": int(e), "G": float(g)}
        for a, b, c, d, e, g in rows
    ]
    out["real_gaunt_dipole_tol"] = 1e-9
    src = read("src/tests/test_gaunt.cpp")
    body = src[src.index("const Triple cases[]"):]
    body = body[: body.index("};")]
    rows = re.findall(r"\{\s*(-?\d+),\s*([+-]?\d+),\s*(-?\d+),\s*([+-]?\d+),\s*(-?\d+),\s*([+-]?\d+)\s*\}", body)
    out["gaunt_permutation_cases"] = [[int(x) for x in r] for r in rows]
    out["gaunt_tol"] = 1e-14
    src = read("src/tests/test_freeparticle_dipole.cpp")
    ks = re.search(r"const double ks\[\] = \{([^}]*)\}", src).group(1)
    out["freeparticle"] = {
        "ks": [float(x) for x in ks.split(",")],
        "Nr": int(re.search(r"const int\s+Nr = (\d+);", src).group(1)),
        "dr": float(re.search(r"const double dr = ([0-9.]+);", src).group(1)),
        "alpha": 1.0,
        "rel_tol_dL": 1e-6,
        "norm_tol": 1e-10,
    }
    with open(os.path.join(HERE, "reference_unit_vectors.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['real_gaunt_dipole'])} real-Gaunt dipole values, "
          f"{len(out['gaunt_permutation_cases'])} permutation cases")


if __name__ == "__main__":
    main()

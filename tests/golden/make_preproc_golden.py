"""Writes tests/golden/preproc_reference.json from the reference's own
preprocessing fixtures (preprocessing/reference_data/ of a checkout of the
reference, given as the argument): for H2 and H2O in cc-pVDZ (spherical),
the Molden file's text and the pointwise values the reference's tests
compare against -- rho and psi_HOMO at 76 points (an independent evaluator
of the same Molden basis; preprocessing/tests/test_basis_pointwise.cpp) and
V_H at 72 points (Psi4's analytic electrostatic potential of the SCF
density; preprocessing/tests/test_v_H_pointwise.cpp).

    python tests/golden/make_preproc_golden.py REFERENCE_CHECKOUT
"""
import json
import os
import sys

if len(sys.argv) < 2:
    sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT")
REF = os.path.join(sys.argv[1], "preprocessing", "reference_data")
out = {}
for name in ("h2_ccpvdz_sph", "h2o_ccpvdz_sph"):
    with open(os.path.join(REF, name + ".molden")) as f:
        text = f.read()
    with open(os.path.join(REF, name + "_reference.json")) as f:
        d = json.load(f)
    pw = d["pointwise_reference"]
    out[name] = {
        "molden": text,
        "nbf": d["nbf"],
        "orbital_energies_hartree": d["orbital_energies_hartree"],
        "occupations": d["occupations"],
        "homo_energy_hartree": pw["homo_energy_hartree"],
        "points_xyz_bohr": pw["points_xyz_bohr_rowmajor"],
        "rho": pw["rho"],
        "psi_homo": pw["psi_homo"],
        "v_H_points_xyz_bohr": pw["v_H"]["points_xyz_bohr_rowmajor"],
        "v_H": pw["v_H"]["V_H_hartree"],
    }
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "preproc_reference.json")
with open(dst, "w") as f:
    json.dump(out, f)
print(dst)

"""The preprocessing chain of the reference (preprocessing/src/
main_preprocess.cpp: Molden file -> single-centre expansion of the
orbitals and the density -> Hartree potential -> the schema-v2 file the
scattering solve reads), on the library's device steps:

    read_molden (scatt_molden_*)  ->  sce_basis (scatt_sce_basis: orbitals,
    density, local exchange)  ->  hartree (scatt_hartree)  ->
    h5io.write_preproc

The SCE origin is placed at (0, 0, 0) and the atoms are translated so that
the chosen centre sits there (main_preprocess.cpp:278-303): 'atoms' (their
geometric mean, the default), 'com' (the Z-weighted mean) or
'origin_of_file'.  The radial grid is r_k = k dr, k = 0 .. round(rmax / dr)
(rmin = 0, as the solver's grid).  The occupied orbitals are the alpha
orbitals with a non-zero occupation, in file order.
"""
from __future__ import annotations

import math
import sys

import numpy as np

from . import _lib, h5io
from .molden import read_molden
from .synth import ScanInputs


def centre_of(atoms: np.ndarray, choice: str) -> np.ndarray:
    """main_preprocess.cpp:283-299."""
    if choice in ("atoms", "auto"):
        return atoms[:, 1:].mean(axis=0)
    if choice == "com":
        return (atoms[:, :1] * atoms[:, 1:]).sum(axis=0) / atoms[:, 0].sum()
    if choice == "origin_of_file":
        return np.zeros(3)
    raise ValueError(f"unknown origin choice {choice!r}")


def simpson_weights(Nr: int, dr: float) -> np.ndarray:
    """Composite Simpson weights on r_k = k dr (Nr odd), the radial rule of
    the reference's density and norm checks (SCE.hpp:268-285)."""
    w = np.full(Nr, 2.0 * dr / 3.0)
    w[1::2] = 4.0 * dr / 3.0
    w[0] = w[-1] = dr / 3.0
    return w


def norm_squared(F_lm: np.ndarray, dr: float) -> float:
    """SCE.hpp:268-276: ||psi||^2 = int r^2 sum_lm F_lm(r)^2 dr."""
    Nr = F_lm.shape[-1]
    r = np.arange(Nr) * dr
    return float(np.sum(simpson_weights(Nr, dr) * r * r * np.sum(F_lm * F_lm, axis=0)))


def inner_product_radial(Fa: np.ndarray, Fb: np.ndarray, dr: float) -> float:
    """Vnuclear.hpp:210-230: <Fa|Fb> = int r^2 sum_lm Fa_lm(r) Fb_lm(r) dr,
    the reference's Coulomb sanity sums (J = 0.5 <rho|V_H>)."""
    if Fa.shape != Fb.shape:
        raise ValueError("inner_product_radial: shape mismatch")
    Nr = Fa.shape[-1]
    r = np.arange(Nr) * dr
    return float(np.sum(simpson_weights(Nr, dr) * r * r * np.sum(Fa * Fb, axis=0)))


def validate(orb_norm_sq, N_e: float, N_e_expected: float, norm_lo: float = 0.50, norm_hi: float = 1.10,
             ne_tol: float = 0.10) -> dict:
    """The input-convention gate of main_preprocess.cpp:557-632: every
    occupied orbital's ||psi||^2 in [norm_lo, norm_hi] and
    |N_e / N_e_expected - 1| <= ne_tol.  Returns {'ok', 'failures' (lines),
    'worst_norm' (lo, hi), 'ne_rel', 'advisory' (norms below 0.99, the
    production criterion the reference names)}."""
    norms = np.asarray(orb_norm_sq, dtype=np.float64)
    fails = [f"orbital {j + 1}: ||psi||^2 = {v:.12g} outside [{norm_lo}, {norm_hi}]"
             for j, v in enumerate(norms) if v < norm_lo or v > norm_hi]
    advisory = int(np.count_nonzero((norms >= norm_lo) & (norms <= norm_hi) & (norms < 0.99)))
    ne_rel = abs(N_e / N_e_expected - 1.0) if N_e_expected > 0.0 else 0.0
    if ne_rel > ne_tol:
        fails.append(f"N_e(SCE rho) = {N_e:.12g} vs occupations {N_e_expected:.12g}: "
                     f"relative error {100 * ne_rel:.4g}% > {100 * ne_tol:.4g}%")
    return {"ok": not fails, "failures": fails,
            "worst_norm": (float(norms.min()) if norms.size else None, float(norms.max()) if norms.size else None),
            "ne_rel": float(ne_rel), "advisory": advisory}


def preprocess(molden_path, Lmax: int, dr: float, rmax: float, origin: str = "atoms", l_cont: int = 0,
               chunk: int = 0, exchange: str = "none"):
    """(ScanInputs, extras): the scan's energy-independent inputs from a
    Molden file -- psi_lm the SCE coefficients of every alpha orbital
    (Lmax channels), V_H from the SCE density by the radial Poisson
    integrals -- and extras {'rho_lm', 'V_x' (with exchange 'slater' or
    'ks'), 'centre', 'N_e', 'N_e_expected', 'orb_norm_sq'}.  N_e =
    sqrt(4 pi) int r^2 rho_00 dr by Simpson's rule, the reference's density
    check (SCE.hpp:278-285); N_e_expected the sum of the alpha and beta
    occupations (main_preprocess.cpp:270-273); orb_norm_sq the ||psi||^2 of
    each occupied alpha orbital's expansion (SCE.hpp:268-276); J the
    Coulomb energy 0.5 <rho|V_H> (main_preprocess.cpp:505-508)."""
    m = read_molden(molden_path)
    atoms = m["atoms"].copy()
    c = centre_of(atoms, origin)
    atoms[:, 1:] -= c
    shells = [(cen - c, l, e, k) for cen, l, e, k in m["shells"]]
    Nr = int(round(rmax / dr)) + 1
    a = m["alpha"]
    vx_form = {"none": 0, "slater": 1, "ks": 2}[exchange]
    out = _lib.sce_basis(shells, a["C"], a["occ"], Lmax, Nr, 0.0, dr, (0.0, 0.0, 0.0), chunk, vx_form=vx_form)
    orb, rho = out[0], out[1]
    if m["beta"]["C"].shape[0]:
        # the beta orbitals' density adds to the alpha one (evaluate_density)
        b = m["beta"]
        rho = rho + _lib.sce_basis(shells, b["C"], b["occ"], Lmax, Nr, 0.0, dr, (0.0, 0.0, 0.0), chunk)[1]
    V_H = _lib.hartree(rho, dr, Lmax)
    r = np.arange(Nr) * dr
    w = simpson_weights(Nr, dr)
    extras = {"rho_lm": rho, "centre": c, "N_e": math.sqrt(4.0 * math.pi) * float(np.sum(w * r * r * rho[0])),
              "N_e_expected": float(np.sum(a["occ"]) + np.sum(m["beta"]["occ"])),
              "orb_norm_sq": [norm_squared(orb[j], dr) for j in np.flatnonzero(a["occ"])],
              "J": 0.5 * inner_product_radial(rho, V_H, dr)}
    if vx_form:
        extras["V_x"] = out[2]
    n_occ = int(np.count_nonzero(a["occ"]))
    inp = ScanInputs(name=str(molden_path), dr=float(dr), Nr=Nr, l_cont=int(l_cont or min(Lmax, 10)),
                     atoms=atoms, psi_lm=orb, orb_energies=a["energy"].copy(), n_occ=n_occ, V_H=V_H)
    return inp, extras


def preprocess_to_file(molden_path, path, Lmax: int, dr: float, rmax: float, split: bool = False, **kw):
    """preprocess() written in the reference's schema (h5io.write_preproc);
    returns the path to open (ScanSolver.from_preproc)."""
    inp, _ = preprocess(molden_path, Lmax, dr, rmax, **kw)
    return h5io.write_preproc(path, inp, split=split)


def main(argv=None):
    """Command line in the manner of the reference's preprocess tool
    (main_preprocess.cpp:60-210: --lmax, --dr, --rmax, --exchange,
    --origin): python -m scatt_b200.preprocess MOLDEN OUT [--split]."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m scatt_b200.preprocess")
    ap.add_argument("molden")
    ap.add_argument("out", help="combined file path, or the stem of the split pair with --split")
    ap.add_argument("--lmax", type=int, default=20)
    ap.add_argument("--dr", type=float, default=0.01)
    ap.add_argument("--rmax", type=float, default=40.0)
    ap.add_argument("--exchange", default="none", choices=["none", "slater", "ks"])
    ap.add_argument("--origin", default="atoms", choices=["atoms", "auto", "com", "origin_of_file"])
    ap.add_argument("--split", action="store_true")
    ap.add_argument("--no-validate-input", dest="validate", action="store_false")
    ap.add_argument("--validate-norm-lo", type=float, default=0.50)
    ap.add_argument("--validate-norm-hi", type=float, default=1.10)
    ap.add_argument("--validate-ne-tol", type=float, default=0.10)
    a = ap.parse_args(argv)
    inp, ex = preprocess(a.molden, a.lmax, a.dr, a.rmax, origin=a.origin, exchange=a.exchange)
    check = None
    if a.validate:
        # main_preprocess.cpp:557-632: a failed gate writes nothing and exits 3
        check = validate(ex["orb_norm_sq"], ex["N_e"], ex["N_e_expected"], a.validate_norm_lo,
                         a.validate_norm_hi, a.validate_ne_tol)
        if not check["ok"]:
            for line in check["failures"]:
                print(f"[validate] FAIL {line}", file=sys.stderr)
            print("[validate] the SCE density is inconsistent with the orbital occupations (a basis-convention "
                  "error in the Molden file?); nothing written.  --no-validate-input skips the check.",
                  file=sys.stderr)
            return 3
    extra = {"/rho/rho_lm": ex["rho_lm"]}
    if "V_x" in ex:
        extra["/potential/V_local_exchange"] = ex["V_x"]
    path = h5io.write_preproc(a.out, inp, split=a.split, extra=extra)
    print(json.dumps({"file": path, "Nr": inp.Nr, "Lmax": a.lmax, "orbitals": int(inp.psi_lm.shape[0]),
                      "n_occ": inp.n_occ, "N_e": ex["N_e"], "N_e_expected": ex["N_e_expected"],
                      "orb_norm_sq": [float(v) for v in ex["orb_norm_sq"]], "J": ex.get("J"),
                      "validate": None if check is None else {k: check[k] for k in ("worst_norm", "ne_rel", "advisory")},
                      "centre": [float(x) for x in ex["centre"]]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())

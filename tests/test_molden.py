"""The library's Molden reader (scatt_molden_*, the parser of
preprocessing/src/molden/Molden.hpp) on seeded files written here: atoms
in bohr and Angstrom, spherical flags, Fortran exponents, alpha and beta
orbitals in any header order, and the reference's errors (missing
sections, bad lines, indices out of range, combined sp shells, Cartesian
d without [5D]).  Host-only: no GPU."""
import numpy as np
import pytest

from scatt_b200 import molden
from scatt_b200._lib import ScattError

BOHR_PER_ANGSTROM = 1.8897261245650618


def molden_text(rng, units="AU", flags="[5D7F]", fortran=False, beta=True):
    atoms = [("O", 8, np.zeros(3)), ("H", 1, np.array([0.0, 1.43, 1.1])), ("H", 1, np.array([0.0, -1.43, 1.1]))]
    shells = {0: [("s", 3), ("s", 1), ("p", 2), ("d", 1)], 1: [("s", 2), ("p", 1)], 2: [("s", 2), ("p", 1)]}
    lines = ["[Molden Format]", f"[Atoms] {units}"]
    for i, (sym, z, x) in enumerate(atoms):
        lines.append(f"{sym:2s} {i + 1} {z} " + " ".join(f"{v:.10f}" for v in x))
    lines.append(flags)
    lines.append("[GTO]")
    prims = []
    num = (lambda v: f"{v:.12E}".replace("E", "D")) if fortran else (lambda v: f"{v:.12E}")
    nbf = 0
    for a in range(3):
        lines.append(f"  {a + 1} 0")
        for letter, n in shells[a]:
            lines.append(f" {letter}   {n} 1.00")
            e, c = rng.uniform(0.1, 9.0, n), rng.uniform(-1.0, 1.0, n)
            prims.append((a, "spdf".index(letter), e, c))
            for ei, ci in zip(e, c):
                lines.append(f"   {num(ei)}  {num(ci)}")
            nbf += 2 * "spdf".index(letter) + 1
        lines.append("")
    lines.append("[MO]")
    mos = []
    for spin in (("Alpha", "Beta") if beta else ("Alpha",)):
        for i in range(3):
            Cv = rng.standard_normal(nbf)
            ene, occ = -1.0 + 0.3 * i, (1.0 if spin == "Beta" else 2.0) if i < 2 else 0.0
            hdr = [f" Sym= A{i}", f" Ene= {num(ene)}", f" Spin= {spin}", f" Occup= {occ:.6f}"]
            lines += hdr[::-1] if i % 2 else hdr
            for k, v in enumerate(Cv):
                if k % 5 != 3:                     # missing entries read as zero
                    lines.append(f"  {k + 1} {num(v)}")
            Cv = np.where(np.arange(nbf) % 5 != 3, Cv, 0.0)
            mos.append((spin, Cv, occ, ene))
    return "\n".join(lines) + "\n", atoms, prims, nbf, mos


@pytest.mark.parametrize("units,fortran", [("AU", False), ("(Angs)", True), ("", False)])
def test_reader_keeps_what_the_file_says(tmp_path, units, fortran):
    rng = np.random.default_rng(21)
    text, atoms, prims, nbf, mos = molden_text(rng, units=units, fortran=fortran)
    p = tmp_path / "m.molden"
    p.write_text(text)
    m = molden.read_molden(p)
    scale = 1.0 if units == "AU" else BOHR_PER_ANGSTROM
    for (sym, z, x), row in zip(atoms, m["atoms"]):
        assert row[0] == z
        np.testing.assert_allclose(row[1:], np.round(x, 10) * scale, rtol=0, atol=1e-12)
    assert m["nbf"] == nbf and len(m["shells"]) == len(prims)
    for (a, l, e, c), (cen, ll, ee, cc) in zip(prims, m["shells"]):
        assert ll == l
        np.testing.assert_allclose(cen, m["atoms"][a, 1:], rtol=0, atol=0)
        np.testing.assert_allclose(ee, e, rtol=1e-12)
        np.testing.assert_allclose(cc, c, rtol=1e-12)
    for spin in ("alpha", "beta"):
        want = [x for x in mos if x[0].lower() == spin]
        assert m[spin]["C"].shape == (len(want), nbf)
        for i, (_, Cv, occ, ene) in enumerate(want):
            np.testing.assert_allclose(m[spin]["C"][i], Cv, rtol=1e-12)
            assert m[spin]["occ"][i] == occ and abs(m[spin]["energy"][i] - ene) <= 1e-12


def test_cartesian_d_needs_the_spherical_flag(tmp_path):
    rng = np.random.default_rng(2)
    text, *_ = molden_text(rng, flags="")
    p = tmp_path / "cart.molden"
    p.write_text(text)
    with pytest.raises(ScattError, match="Cartesian"):
        molden.read_molden(p)


@pytest.mark.parametrize("edit,msg", [
    (lambda t: t.replace("[GTO]", "[GTX]"), r"\[gto\] section missing"),
    (lambda t: t.replace("[MO]", "[MQ]"), r"\[mo\] section missing"),
    (lambda t: t.replace("  2 0", "  7 0"), "atom index out of range"),
    (lambda t: t.replace(" p   1 1.00", " sp   1 1.00", 1), "combined 'sp'"),
    (lambda t: t.replace(" Ene= ", " Ene= x", 1), "does not parse"),
    (lambda t: t + "  999 1.0\n", "index out of range"),
])
def test_malformed_files_are_io_errors(tmp_path, edit, msg):
    rng = np.random.default_rng(3)
    text, *_ = molden_text(rng)
    p = tmp_path / "bad.molden"
    p.write_text(edit(text))
    with pytest.raises(ScattError, match=msg) as ei:
        molden.read_molden(p)
    assert ei.value.code == 11                     # SCATT_ERR_IO


def test_missing_file_is_an_io_error(tmp_path):
    with pytest.raises(ScattError) as ei:
        molden.read_molden(tmp_path / "none.molden")
    assert ei.value.code == 11


def test_sce_centre_choices():
    """main_preprocess.cpp:283-299: the geometric mean of the atoms, the
    Z-weighted mean, or the file's own origin."""
    from scatt_b200 import preprocess
    atoms = np.array([[8.0, 0.0, 0.0, 0.0], [1.0, 0.0, 1.43, 1.1], [1.0, 0.0, -1.43, 1.1]])
    np.testing.assert_allclose(preprocess.centre_of(atoms, "atoms"), [0.0, 0.0, 2.2 / 3.0], atol=1e-15)
    np.testing.assert_allclose(preprocess.centre_of(atoms, "com"), [0.0, 0.0, 2.2 / 10.0], atol=1e-15)
    assert np.array_equal(preprocess.centre_of(atoms, "origin_of_file"), np.zeros(3))
    with pytest.raises(ValueError):
        preprocess.centre_of(atoms, "elsewhere")

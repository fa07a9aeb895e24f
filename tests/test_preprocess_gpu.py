"""The preprocessing chain on the device (scatt_b200.preprocess: Molden file
-> single-centre expansion of the orbitals and the density -> Hartree
potential -> the reference's schema-v2 file), and the scattering solve on
the file it writes.

The orbitals are made orthonormal first, against the AO overlap that the
expansion grid itself integrates (the angular quadrature times Simpson's
rule in r, on the oracle's AO values), by Loewdin's orthonormalisation.
Checked: the chain against the oracle's (oracle/basis.py, oracle/sce.py,
oracle/hartree.py) -- psi_lm and rho_lm to 1e-12, V_H within 1e-12 plus the
Hartree formula's summation floor (tests/test_hartree_gpu.py); the density
integrates to the occupations' electron count (the same quadrature that
made the orbitals orthonormal: to 1e-10); a solve from the written file
equals the solve from the same inputs in memory (K bit for bit, the
dipoles to rounding)."""
import math

import numpy as np
import pytest

import test_hartree_gpu as TH
import test_molden as TM
from oracle import basis as B
from oracle import hartree as H
from oracle import sce as SC
from scatt_b200 import _lib, preprocess
from scatt_b200 import solver as S

pytestmark = pytest.mark.gpu


def _orthonormal_molden(path, Lmax, dr, rmax):
    """A seeded Molden file whose alpha orbitals are orthonormal on the grid."""
    rng = np.random.default_rng(40)
    text, atoms, prims, nbf, mos = TM.molden_text(rng, beta=False)
    p = path / "raw.molden"
    p.write_text(text)
    m = preprocess.read_molden(p)
    c = preprocess.centre_of(m["atoms"], "atoms")
    shells = [(cen - c, l, e, k) for cen, l, e, k in m["shells"]]
    Nr = int(round(rmax / dr)) + 1
    r = np.arange(Nr) * dr
    w = np.full(Nr, 2.0 * dr / 3.0)
    w[1::2] = 4.0 * dr / 3.0
    w[0] = w[-1] = dr / 3.0
    _, wq, _, phi = SC.grid(Lmax)
    chi = B.ao_values(shells, B.grid_points(Lmax, r, np.zeros(3))).reshape(nbf, Nr, Lmax + 1, phi.size)
    Sao = (2.0 * math.pi / phi.size) * np.einsum("akij,bkij,k,i->ab", chi, chi, w * r * r, wq)
    Cm = m["alpha"]["C"]
    ev, U = np.linalg.eigh(Cm @ Sao @ Cm.T)
    Cn = (U @ np.diag(ev ** -0.5) @ U.T) @ Cm
    lines = text.splitlines()
    i0 = lines.index("[MO]")
    out = lines[:i0 + 1]
    for i in range(Cn.shape[0]):
        occ = m["alpha"]["occ"][i]
        out += [f" Sym= A{i}", f" Ene= {m['alpha']['energy'][i]:.12E}", " Spin= Alpha", f" Occup= {occ:.6f}"]
        out += [f"  {j + 1} {Cn[i, j]:.16E}" for j in range(nbf)]
    q = path / "orth.molden"
    q.write_text("\n".join(out) + "\n")
    return q, shells, Cn, m["alpha"]["occ"]


def test_preprocessing_chain_matches_oracle_and_feeds_the_solver(tmp_path):
    Lmax, dr, rmax = 8, 0.05, 15.0
    path, shells, Cn, occ = _orthonormal_molden(tmp_path, Lmax, dr, rmax)
    inp, ex = preprocess.preprocess(path, Lmax, dr, rmax)
    Nr = inp.Nr
    r = np.arange(Nr) * dr
    orb_ref, rho_ref = B.sce_of_basis(shells, Cn, occ, Lmax, r, np.zeros(3))
    for i in range(Cn.shape[0]):
        assert np.max(np.abs(inp.psi_lm[i] - orb_ref[i])) <= 1e-12 * np.max(np.abs(orb_ref[i]))
    assert np.max(np.abs(ex["rho_lm"] - rho_ref)) <= 1e-12 * np.max(np.abs(rho_ref))
    vh_ref = H.build_V_H(rho_ref, dr, Lmax)
    fl = TH.summation_floor(rho_ref, dr, Lmax)
    for ch in range(vh_ref.shape[0]):
        scale = max(np.max(np.abs(vh_ref[ch])), 1e-300)
        # rho differs from the oracle's by 1e-12 relative: the floor takes that too
        assert np.all(np.abs(inp.V_H[ch] - vh_ref[ch]) <= 1e-10 * scale + fl[ch]), ch
    assert abs(ex["N_e"] - occ.sum()) <= 1e-10 * occ.sum()
    # the file the chain writes, solved, equals the in-memory inputs solved
    f = preprocess.h5io.write_preproc(tmp_path / "mol.h5", inp)
    a = S.ScanSolver(inp)
    b = S.ScanSolver.from_preproc(f, l_cont_max=inp.l_cont)
    o = S.default_opts(allow_closed_channels=1)
    Es = [0.3, 0.8]
    ra, rb = a.solve(Es, opts=o), b.solve(Es, opts=o)
    for x, y in zip(ra, rb):
        assert x.status == 0 and y.status == 0
        assert np.array_equal(x.K_kme, y.K_kme)
        # each solver builds its own dipole tables, whose d_correction sums
        # run in shared-memory atomic order: equal to rounding
        assert np.max(np.abs(x.D - y.D)) <= 1e-10 * np.max(np.abs(x.D))
        assert np.all(np.isfinite(x.K_kme))
        assert np.max(np.abs(x.K_kme - x.K_kme.T)) <= 1e-8 * np.max(np.abs(x.K_kme))
    a.close()
    b.close()

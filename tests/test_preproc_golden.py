"""The preprocessing oracle against the reference's own fixtures
(tests/golden/preproc_reference.json, written by make_preproc_golden.py from
preprocessing/reference_data/): the Molden files of H2 and H2O in cc-pVDZ
read by the library's reader, the oracle's basis (oracle/basis.py: the
normalisation and molden order of MoldenBasis.hpp) evaluated at the
reference's 76 points against its rho and psi_HOMO -- the check of
preprocessing/tests/test_basis_pointwise.cpp, 1e-12 absolute -- and the
oracle's SCE + Hartree chain synthesised at the reference's 72 points
against Psi4's analytic electrostatic potential of the same density -- the
check of preprocessing/tests/test_v_H_pointwise.cpp, Lmax 40, dr 0.0025,
R 15, 5e-5 hartree.  The device steps are held to these oracles by the GPU
tests (test_sce_basis_gpu.py, test_hartree_gpu.py, test_preprocess_gpu.py)."""
import json
import os

import numpy as np
import pytest

from oracle import basis as B
from oracle import hartree as H
from oracle import sce as SC
from scatt_b200 import molden

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "preproc_reference.json")


@pytest.fixture(scope="module")
def gold():
    with open(GOLD) as f:
        return json.load(f)


def _read(g, name, tmp_path):
    p = tmp_path / (name + ".molden")
    p.write_text(g[name]["molden"])
    return molden.read_molden(p)


def _homo_and_occupied(m):
    a = m["alpha"]
    occ = a["occ"]
    homo = max((i for i in range(occ.size) if occ[i] > 0), key=lambda i: a["energy"][i])
    return homo, a["C"][occ > 0], occ[occ > 0]


@pytest.mark.parametrize("name", ["h2_ccpvdz_sph", "h2o_ccpvdz_sph"])
def test_basis_pointwise_matches_reference(gold, tmp_path, name):
    g = gold[name]
    m = _read(gold, name, tmp_path)
    assert m["nbf"] == g["nbf"]
    np.testing.assert_allclose(m["alpha"]["energy"], g["orbital_energies_hartree"], rtol=0, atol=1e-10)
    np.testing.assert_array_equal(m["alpha"]["occ"], g["occupations"])
    homo, C_occ, occ = _homo_and_occupied(m)
    assert abs(m["alpha"]["energy"][homo] - g["homo_energy_hartree"]) <= 1e-10
    pts = np.asarray(g["points_xyz_bohr"]).reshape(-1, 3)
    chi = B.ao_values(m["shells"], pts)
    psi_homo = m["alpha"]["C"][homo] @ chi
    rho = occ @ (C_occ @ chi) ** 2
    assert np.max(np.abs(psi_homo - np.asarray(g["psi_homo"]))) <= 1e-12
    assert np.max(np.abs(rho - np.asarray(g["rho"]))) <= 1e-12


def test_hartree_chain_pointwise_matches_psi4(gold, tmp_path):
    g = gold["h2_ccpvdz_sph"]
    m = _read(gold, "h2_ccpvdz_sph", tmp_path)
    _, C_occ, occ = _homo_and_occupied(m)
    origin = m["atoms"][:, 1:].mean(axis=0)
    Lmax, dr, R = 40, 0.0025, 15.0
    Nr = int(round(R / dr)) + 1
    r = np.arange(Nr) * dr
    nt, n_phi = Lmax + 1, 2 * (Lmax + 1)
    samples = np.empty((Nr, nt, n_phi))
    for k0 in range(0, Nr, 400):                         # the density on the grid, in radial chunks
        k1 = min(Nr, k0 + 400)
        chi = B.ao_values(m["shells"], B.grid_points(Lmax, r[k0:k1], origin))
        samples[k0:k1] = (occ @ (C_occ @ chi) ** 2).reshape(k1 - k0, nt, n_phi)
    rho_lm = SC.project(samples, Lmax)
    V = H.build_V_H(rho_lm, dr, Lmax)
    P = np.asarray(g["v_H_points_xyz_bohr"]).reshape(-1, 3)
    got = np.array([SC.synthesize_at(V, 0.0, dr, origin, Lmax, p) for p in P])
    assert np.max(np.abs(got - np.asarray(g["v_H"]))) <= 5e-5

"""The oracle's channel potential V(r) (oracle.potentials.VCube, restating
Potentials::build / V_at) against the reference's potential test and an
exact property of the multipole expansion.

src/tests/test_potential_h2o.cpp: (1) V symmetric at every radius
(1e-10), (2) at r = r(N - 2) the diagonal within 5 mHa of l (l + 1) / (2 r^2)
and every off-diagonal element below 5 mHa.  The synthetic H2O-like input
carries only the L = 0 Hartree multipole, so the nuclear dipole of the two
H centres is not screened as in the molecule, and at the reference's
r_max = 15 bohr its tail (5.7 mHa) exceeds the allowance.  The check is
made at r_max = 30 bohr.

Exactness: the matrix element <Y_mu| f |Y_nu> of l_mu, l_nu <= l_cont only
involves multipoles L <= 2 l_cont, which is where Potentials.cpp:40-88
truncates the expansion of the nuclear attraction.  So V(r) minus the
centrifugal term must equal the quadrature over the sphere of
-sum_A Z_A / |r - R_A| + sum_sigma V_H,sigma(r) Y_sigma times Y_mu Y_nu,
to quadrature accuracy, for any atom positions.
"""
import math

import numpy as np

from oracle import angular as A
from oracle.potentials import VCube
from scatt_b200 import synth
from scatt_b200.synth import ScanInputs, lm_to_idx


def test_potential_checks():
    inp = synth.h2o_like(Nr=601, dr=0.05, l_cont=6, lmax_orb=6, n_orb=5)
    vc = VCube(inp)
    assert max(np.max(np.abs(vc.get(ir) - vc.get(ir).T)) for ir in range(inp.Nr)) < 1e-10
    ir = inp.Nr - 2
    r = ir * inp.dr
    V = vc.get(ir)
    l = vc.cent
    assert np.max(np.abs(np.diag(V) - l * (l + 1.0) / (2.0 * r * r))) < 5e-3
    assert np.max(np.abs(V - np.diag(np.diag(V)))) < 5e-3


def test_multipole_potential_equals_sphere_quadrature():
    Nr, dr, l_cont = 401, 0.05, 4
    r_grid = np.arange(Nr) * dr
    atoms = np.array([[8.0, 0.0, 0.0, 0.0],
                      [1.0, 1.43, 0.0, 1.11],
                      [1.0, -0.7, 1.2, -0.4]])
    VH = np.zeros((4, Nr))                     # Hartree multipoles L = 0 and L = 1 (m = 0)
    VH[lm_to_idx(0, 0)] = 8.0 * np.exp(-0.3 * r_grid)
    VH[lm_to_idx(1, 0)] = 0.7 * r_grid * np.exp(-0.5 * r_grid)
    inp = ScanInputs(name="three_centres", dr=dr, Nr=Nr, l_cont=l_cont, atoms=atoms,
                     psi_lm=np.zeros((1, 1, Nr)), orb_energies=np.array([-0.5]), n_occ=1, V_H=VH)
    vc = VCube(inp)

    n_theta, n_phi = 96, 192
    ct, w = np.polynomial.legendre.leggauss(n_theta)
    TH, PH = np.meshgrid(np.arccos(ct), np.arange(n_phi) * 2.0 * math.pi / n_phi, indexing="ij")
    weight = w[:, None] * (2.0 * math.pi / n_phi)
    ylm = np.vectorize(A.real_Ylm)
    ch = (l_cont + 1) ** 2
    Y = np.stack([ylm(*A.idx_to_lm(mu), TH, PH) for mu in range(ch)])
    Y10 = ylm(1, 0, TH, PH)
    ux, uy, uz = np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)

    # radii away from the centres (|R| = 1.81 and 1.45), where the integrand is smooth
    for ir in (10, 20, 100, 300):
        r = ir * dr
        f = VH[0, ir] / math.sqrt(4.0 * math.pi) + VH[lm_to_idx(1, 0), ir] * Y10
        for Z, x, y, z in atoms:
            f = f - Z / np.sqrt((r * ux - x) ** 2 + (r * uy - y) ** 2 + (r * uz - z) ** 2)
        Vq = np.einsum("aij,bij,ij->ab", Y, Y, f * weight)
        Vo = vc.get(ir) - np.diag(vc.cent * (vc.cent + 1.0) * 0.5 / (r * r))
        assert np.max(np.abs(Vq - Vo)) < 1e-12 * np.max(np.abs(Vq))

"""The oracle's contracted spherical-Gaussian basis (oracle/basis.py,
restating preprocessing/src/basis/MoldenBasis.hpp and SphericalGaussian.hpp)
against properties the reference states: every normalised AO has unit norm
(SphericalGaussian.hpp:1-40; here by the single-centre expansion of AOs at
the origin and Simpson's rule in r), the molden order of a shell's
components (MoldenBasis.hpp:110-127), and a p_z AO landing in the (1, 0)
channel alone."""
import math

import numpy as np
import pytest

from oracle import basis as B
from oracle import sce as SC


def test_molden_component_order():
    assert [B.molden_m(1, i) for i in range(3)] == [1, -1, 0]
    assert [B.molden_m(2, i) for i in range(5)] == [0, 1, -1, 2, -2]
    assert [B.molden_m(3, i) for i in range(7)] == [0, 1, -1, 2, -2, 3, -3]


@pytest.mark.parametrize("l", [0, 1, 2, 3])
def test_centred_aos_are_normalised(l):
    shells = [(np.zeros(3), l, [0.35, 1.3, 4.0], [0.4, 0.5, 0.3])]
    Lmax = l + 1
    dr = 0.005
    r = np.arange(2401) * dr                             # 0 .. 12 bohr, an odd count for Simpson
    pts = B.grid_points(Lmax, r, np.zeros(3))
    chi = B.ao_values(shells, pts)
    shape = (r.size, Lmax + 1, 2 * (Lmax + 1))
    w = np.full(r.size, 2.0)
    w[1::2] = 4.0
    w[0] = w[-1] = 1.0
    w *= dr / 3.0
    for mu in range(chi.shape[0]):
        F = SC.project(chi[mu].reshape(shape), Lmax)
        norm = float(np.sum(w * r ** 2 * np.sum(F ** 2, axis=0)))
        assert abs(norm - 1.0) <= 1e-8, (l, mu, norm)
        m = B.molden_m(l, mu)
        ch = l * l + l + m
        assert np.max(np.abs(np.delete(F, ch, axis=0))) <= 1e-12 * np.max(np.abs(F[ch]))


def test_contraction_scale_matches_closed_form_for_one_primitive():
    for l in range(4):
        for a in (0.3, 2.0):
            assert math.isclose(B.c_tilde(l, [a], [1.0])[0], B.n_sph(a, l), rel_tol=1e-14)

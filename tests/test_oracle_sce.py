"""The oracle's single-centre expansion (oracle/sce.py, restating
preprocessing/src/sce/SCE.hpp:122-266 on the grid of angular/Grid.hpp)
against closed forms and exactness: the S_{l,m} values the reference's own
Legendre comments state (angular/Legendre.hpp:30-31), scipy's normalised
Legendre functions, and the exact recovery of band-limited coefficients
(the tensor grid integrates Y^R_lm Y^R_l'm' exactly for l, l' <= Lmax,
Grid.hpp:1-20)."""
import math

import numpy as np
from scipy.special import sph_harm_y

from oracle import sce as SC


def test_s_closed_forms():
    th = np.linspace(0.05, 3.0, 7)
    S = SC.s_table(2, th)
    assert np.allclose(S[0, 0], 1.0 / math.sqrt(4.0 * math.pi), rtol=0, atol=1e-16)
    assert np.allclose(S[1, 0], math.sqrt(3.0 / (4.0 * math.pi)) * np.cos(th), rtol=1e-15, atol=1e-16)
    assert np.allclose(S[1, 1], math.sqrt(3.0 / (8.0 * math.pi)) * np.sin(th), rtol=1e-15, atol=1e-16)
    assert np.allclose(S[2, 2], math.sqrt(15.0 / (32.0 * math.pi)) * np.sin(th) ** 2, rtol=1e-15, atol=1e-16)


def test_s_against_scipy_without_condon_shortley():
    th = np.linspace(0.01, 3.13, 11)
    L = 12
    S = SC.s_table(L, th)
    for l in range(L + 1):
        for m in range(l + 1):
            ref = (-1.0) ** m * np.real(sph_harm_y(l, m, th, 0.0))
            assert np.max(np.abs(S[l, m] - ref)) <= 1e-13, (l, m)


def test_band_limited_coefficients_are_recovered():
    rng = np.random.default_rng(5)
    for Lmax, Lf in ((4, 4), (7, 5), (10, 10)):
        coef = rng.standard_normal(((Lf + 1) ** 2, 3))
        samples = SC.synthesize(coef, Lmax)
        got = SC.project(samples, Lmax)
        want = np.zeros(((Lmax + 1) ** 2, 3))
        want[:coef.shape[0]] = coef
        assert np.max(np.abs(got - want)) <= 1e-13, (Lmax, Lf)


def test_grid_integrates_products_exactly():
    Lmax = 6
    x, w, theta, phi = SC.grid(Lmax)
    assert np.all(np.diff(x) > 0) and abs(w.sum() - 2.0) < 1e-14
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    dphi = 2.0 * math.pi / phi.size
    Y = []
    for ch in range((Lmax + 1) ** 2):
        l = math.isqrt(ch)
        Y.append(np.stack([SC.real_ylm(l, ch - l * l - l, TH[i], PH[i]) for i in range(theta.size)]))
    Y = np.array(Y)
    G = dphi * np.einsum("aij,bij,i->ab", Y, Y, w)
    assert np.max(np.abs(G - np.eye(G.shape[0]))) <= 1e-13

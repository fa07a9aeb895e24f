"""The oracle's real Gaunt coefficients against quadrature, up to l = 50.

src/tests/test_real_gaunt_full_l50.cpp compares gaunt_real(l_mu, m_mu; 1, q;
l_nu, m_nu) with a numerical integral of three real_Ylm on a Gauss-Legendre
(cos theta, N_theta = max(96, 2 L + 8)) x trapezoid (phi, N_phi =
max(192, 4 L)) grid, for every l_mu, l_nu <= 50 with |l_mu - l_nu| = 1, every
m and q in {-1, 0, 1}, and fails a triple when |err| > 5e-7 and (|G| <= 1e-6
or the relative error > 1e-4).

Here the same grid and the same triples.  real_Ylm is Theta_{l|m|}(theta)
times 1, sqrt 2 cos(m phi) or sqrt 2 sin(|m| phi) (Gaunt.hpp:171-181), so on a
product grid the triple integral factors into a theta sum and a phi sum,
which makes all 1.03 million triples cheap.  The factorisation is tied to
real_Ylm itself by a point check.  The analytic coefficient is evaluated
where oracle.angular.m3_candidates allows a nonzero value; everywhere else
the quadrature must vanish, which shows that pruning to those m is exact.
The library's host-side scatt_gaunt_real, which builds the device tables,
is held to the same quadrature.
"""
import math

import numpy as np
import pytest

from oracle import angular as A
from scatt_b200 import _lib

L_MAX = 50


def _phi_factor(m, phi):
    if m == 0:
        return np.ones_like(phi)
    if m > 0:
        return math.sqrt(2.0) * np.cos(m * phi)
    return math.sqrt(2.0) * np.sin(-m * phi)


@pytest.fixture(scope="module")
def quadrature():
    """(triples allowed by m3_candidates with their quadrature values,
    number of triples, largest quadrature value among the pruned ones)."""
    n_theta, n_phi = max(96, 2 * L_MAX + 8), max(192, 4 * L_MAX)
    ct, wct = np.polynomial.legendre.leggauss(n_theta)
    theta = np.arccos(ct)
    dphi = 2.0 * math.pi / n_phi
    phi = np.arange(n_phi) * dphi

    Th = np.zeros((L_MAX + 1, L_MAX + 1, n_theta))
    for l in range(L_MAX + 1):
        for m in range(l + 1):
            Th[l, m] = [A.sph_legendre_noCS(l, m, x) for x in theta]
    Ph = np.stack([_phi_factor(m, phi) for m in range(-L_MAX, L_MAX + 1)])   # row m + L_MAX

    # the factorised form is real_Ylm
    rng = np.random.default_rng(50)
    for l, m in ((0, 0), (1, -1), (7, 5), (23, -17), (50, 50), (50, -1)):
        i, j = int(rng.integers(n_theta)), int(rng.integers(n_phi))
        y = A.real_Ylm(l, m, theta[i], phi[j])
        assert abs(y - Th[l, abs(m), i] * Ph[m + L_MAX, j]) <= 1e-14 * max(abs(y), 1e-300)

    allowed_triples = []
    compared = 0
    max_pruned = 0.0
    for lmu in range(L_MAX + 1):
        for mmu in range(-lmu, lmu + 1):
            for q in (-1, 0, 1):
                phi_int = Ph @ (Ph[mmu + L_MAX] * Ph[q + L_MAX]) * dphi           # over m_nu
                w = wct * Th[lmu, abs(mmu)] * Th[1, abs(q)]
                for lnu in (lmu - 1, lmu + 1):
                    if lnu < 0 or lnu > L_MAX:
                        continue
                    theta_int = Th[lnu, : lnu + 1] @ w                            # over |m_nu|
                    ms = np.arange(-lnu, lnu + 1)
                    Gn = theta_int[np.abs(ms)] * phi_int[ms + L_MAX]
                    allowed = set(A.m3_candidates(mmu, q, lnu))
                    compared += ms.size
                    for k, mnu in enumerate(ms):
                        if int(mnu) in allowed:
                            allowed_triples.append((lmu, mmu, q, lnu, int(mnu), float(Gn[k])))
                        else:
                            max_pruned = max(max_pruned, abs(Gn[k]))
    return allowed_triples, compared, max_pruned


def test_pruned_m_triples_vanish(quadrature):
    triples, compared, max_pruned = quadrature
    assert compared == 1029900
    assert len(triples) > 40000
    assert max_pruned < 1e-14


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_real_gaunt_dipole_channel_to_l50(quadrature, impl):
    g = A.gaunt_real if impl == "oracle" else _lib.lib().scatt_gaunt_real
    triples, _, _ = quadrature
    failed = 0
    max_abs = 0.0
    for lmu, mmu, q, lnu, mnu, Gn in triples:
        Ga = g(lmu, mmu, 1, q, lnu, mnu)
        err = abs(Ga - Gn)
        max_abs = max(max_abs, err)
        rel = err / max(abs(Ga), abs(Gn), 1e-30)
        if err > 5e-7 and (abs(Ga) <= 1e-6 or rel > 1e-4):
            failed += 1
    assert failed == 0
    assert max_abs < 1e-12

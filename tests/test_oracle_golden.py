"""Pins the oracle (and the library's host-side angular / Riccati routines)
to the golden vectors of the reference's own unit tests and to mpmath.

Reference tests restated: src/tests/test_gaunt.cpp, test_real_gaunt_dipole.cpp,
test_freeparticle_dipole.cpp, test_dipole_matrix_element.cpp:80-113 and its
isotropy sum rule (:156-196).
"""
import json
import math
import os
import random

import mpmath
import numpy as np
import pytest

from oracle import angular, bessel, solver
from scatt_b200 import _lib

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_unit_vectors.json")))
INV_SQRT_4PI = 1.0 / math.sqrt(4.0 * math.pi)
SQRT_4PI_3 = math.sqrt(4.0 * math.pi / 3.0)


def implementations():
    lib = _lib.lib()
    return {"oracle": (angular.gaunt_real, angular.angular_dipole, angular.velocity_coef),
            "library": (lib.scatt_gaunt_real, lib.scatt_angular_dipole, lib.scatt_velocity_coef)}


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_gaunt_identities(impl):
    g, _, _ = implementations()[impl]
    tol = GOLD["gaunt_tol"]
    assert abs(g(0, 0, 0, 0, 0, 0) - INV_SQRT_4PI) <= tol
    for l in range(4):
        for m in range(-l, l + 1):
            assert abs(g(l, m, l, m, 0, 0) - INV_SQRT_4PI) <= tol
    for c in GOLD["gaunt_permutation_cases"]:
        l1, m1, l2, m2, l3, m3 = c
        g123 = g(l1, m1, l2, m2, l3, m3)
        assert abs(g(l2, m2, l1, m1, l3, m3) - g123) <= tol
        assert abs(g(l1, m1, l3, m3, l2, m2) - g123) <= tol
        assert abs(g(l3, m3, l2, m2, l1, m1) - g123) <= tol
    assert g(1, 0, 1, 0, 1, 0) == 0.0          # odd parity
    assert g(1, 0, 1, 0, 4, 0) == 0.0          # triangle


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_real_gaunt_dipole_table(impl):
    _, ad, _ = implementations()[impl]
    for t in GOLD["real_gaunt_dipole"]:
        got = ad(t["l_mu"], t["m_mu"], t["q"], t["l_nu"], t["m_nu"])
        assert abs(got - SQRT_4PI_3 * t["G"]) < GOLD["real_gaunt_dipole_tol"], t


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_angular_dipole_and_velocity_coef(impl):
    _, ad, vc = implementations()[impl]
    for q in (-1, 0, 1):
        assert abs(ad(1, q, q, 0, 0) - 1.0 / math.sqrt(3.0)) < 1e-12
    assert abs(ad(0, 0, 0, 0, 0)) < 1e-12
    assert abs(ad(2, 0, 0, 0, 0)) < 1e-12
    assert abs(ad(1, 1, 0, 0, 0)) < 1e-12
    assert abs(ad(1, 0, 1, 0, 0)) < 1e-12
    for (lm, ln, want) in [(1, 0, -1.0), (2, 1, -2.0), (0, 1, 1.0), (1, 2, 2.0), (0, 0, 0.0)]:
        assert vc(lm, ln) == want


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_angular_dipole_isotropy_sum_rule(impl):
    """test_dipole_matrix_element.cpp (3): at fixed l_nu the sum over m_nu, l_mu
    = l_nu +- 1 and m_mu of |A(l_mu m_mu; q; l_nu m_nu)|^2 is the same for
    q = -1, 0, 1 (to 1e-12); there for l_nu <= 3, here up to 12."""
    _, ad, _ = implementations()[impl]
    for l_nu in range(13):
        sums = []
        for q in (-1, 0, 1):
            s = 0.0
            for m_nu in range(-l_nu, l_nu + 1):
                for l_mu in (l_nu - 1, l_nu + 1):
                    if l_mu < 0:
                        continue
                    for m_mu in range(-l_mu, l_mu + 1):
                        s += ad(l_mu, m_mu, q, l_nu, m_nu) ** 2
            sums.append(s)
        assert max(sums) - min(sums) < 1e-12


def test_wigner3j_library_matches_exact():
    lib = _lib.lib()
    rng = random.Random(5)
    worst = 0.0
    for _ in range(2000):
        j1, j2 = rng.randint(0, 40), rng.randint(0, 40)
        j3 = rng.randint(abs(j1 - j2), j1 + j2)
        m1, m2 = rng.randint(-j1, j1), rng.randint(-j2, j2)
        if abs(m1 + m2) > j3:
            continue
        a = lib.scatt_wigner3j(j1, j2, j3, m1, m2, -m1 - m2)
        b = angular.wigner3j(j1, j2, j3, m1, m2, -m1 - m2)
        if b != 0.0:
            worst = max(worst, abs(a - b) / abs(b))
        else:
            assert a == 0.0 or abs(a) < 1e-15
    assert worst < 1e-14


def _mp_riccati(l, x, kind):
    with mpmath.workdps(40):
        f = mpmath.besselj if kind == "j" else mpmath.bessely
        return float(x * mpmath.sqrt(mpmath.pi / (2 * x)) * f(l + mpmath.mpf(1) / 2, x))


@pytest.mark.parametrize("kind", ["j", "y"])
def test_riccati_against_mpmath(kind):
    lib = _lib.lib()
    fl = lib.scatt_riccati_j if kind == "j" else lib.scatt_riccati_y
    fo = bessel.riccati_j if kind == "j" else bessel.riccati_y
    worst_lib = worst_or = 0.0
    for l in [0, 1, 2, 3, 5, 8, 12, 20, 30, 40, 60]:
        for x in [1e-3, 0.01, 0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 20.0, 40.0, 80.0, 120.0, 200.0]:
            ref = _mp_riccati(l, x, kind)
            if ref == 0.0 or not math.isfinite(ref) or abs(ref) < 1e-290 or abs(ref) > 1e290:
                continue
            worst_lib = max(worst_lib, abs(fl(l, x) - ref) / abs(ref))
            worst_or = max(worst_or, abs(fo(l, x) - ref) / abs(ref))
    assert worst_lib < 1e-13
    assert worst_or < 1e-13


def test_freeparticle_dipole_golden():
    """test_freeparticle_dipole.cpp: Simpson normalisation and analytic d^L(k)."""
    fp = GOLD["freeparticle"]
    Nr, dr, a = fp["Nr"], fp["dr"], fp["alpha"]
    r = np.arange(Nr) * dr
    chi = r * np.exp(-0.5 * a * r * r)
    num = solver.simpson(chi * chi, dr)
    ana = math.sqrt(math.pi) / (4.0 * a ** 1.5)
    assert abs(num - ana) / ana < fp["norm_tol"]
    A_ang = angular.angular_dipole(1, 0, 0, 0, 0)
    worst = 0.0
    for k in fp["ks"]:
        psi = bessel.riccati_j(1, k * r)
        dL = solver.simpson(r * psi * (A_ang * chi), dr)
        ref = A_ang * math.sqrt(math.pi / 2.0) * k * k * math.exp(-0.5 * k * k)
        worst = max(worst, abs(dL - ref) / abs(ref))
    assert worst < fp["rel_tol_dL"]


def test_simpson_rule_cases():
    """Exact for cubics for every count DipoleMatrixElement can use (n >= 5).

    n = 4 is excluded on purpose: the reference's stitched rule evaluates
    simpson_one_third(1) there, which counts f[0] twice
    (DipoleMatrixElement.cpp:174-176); the restatement keeps that.
    """
    h = 0.1
    x = np.arange(4) * h
    f = x ** 3 - 2 * x + 1.0
    assert abs(solver.simpson(f, h) - ((3.0 * h / 8.0) * (f[0] + 3 * f[1] + 3 * f[2] + f[3]) + 2.0 * f[0] * h / 3.0)) < 1e-15
    for n in (3, 5, 6, 7, 10, 11):
        x = np.arange(n) * h
        f = x ** 3 - 2 * x + 1.0
        exact = ((x[-1] ** 4) / 4 - x[-1] ** 2 + x[-1])
        got = solver.simpson(f, h)
        assert abs(got - exact) < 1e-12

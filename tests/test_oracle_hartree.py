"""The Hartree potential of the preprocessing step (oracle/hartree.py) against
closed forms and independent quadrature.

- The cumulative integrator is exact for quadratics, and a forward step
  followed by the backward stencil is Simpson's rule (RadialGrid.hpp:63-83).
  Its global order is three, not the four its comment states: each
  one-sided interval leaves h^4 times the third derivative / 24, and the
  error falls 8-fold per halving of h.
- Hydrogen 1s density rho = exp(-2r) / pi, whose potential is
  V(r) = 1/r - (1 + 1/r) exp(-2r) with rho_00 = sqrt(4 pi) rho and
  V_00 = sqrt(4 pi) V: within 2e-6 at dr = 0.01 (7e-7 at r = 0, where
  V(0) = 1), with third-order convergence.
- An l = 2 channel, rho_20 = r^2 exp(-r), against scipy quadrature of
  the two defining integrals.
- The guards: empty channels stay 0, and channels above the overflow-safe
  l stay 0.
"""
import math

import numpy as np
from scipy.integrate import quad

from oracle import hartree as H


def test_cumulative_integrator():
    dr = 0.1
    r = np.arange(41) * dr
    f = 3.0 * r ** 2 - r + 2.0
    I = H.cumulative_integrate(f, dr)
    exact = r ** 3 - 0.5 * r ** 2 + 2.0 * r
    assert np.max(np.abs(I - exact)) < 1e-12
    g3 = np.array([1.0, 0.7, -0.2])
    assert abs(H.cumulative_integrate(g3, dr)[2] - dr / 3.0 * (g3[0] + 4 * g3[1] + g3[2])) < 1e-15
    errs = []
    for h in (0.01, 0.005):
        x = np.arange(int(round(10 / h)) + 1) * h
        g = np.exp(-x) * np.cos(3 * x)
        exact_g = (np.exp(-x) * (3 * np.sin(3 * x) - np.cos(3 * x)) + 1.0) / 10.0
        errs.append(np.max(np.abs(H.cumulative_integrate(g, h) - exact_g)))
    assert 7.0 < errs[0] / errs[1] < 9.0                        # third order


def _hydrogen_error(dr):
    Nr = int(round(40 / dr)) + 1
    r = np.arange(Nr) * dr
    rho = np.zeros((1, Nr))
    rho[0] = math.sqrt(4 * math.pi) * np.exp(-2 * r) / math.pi
    V = H.build_V_H(rho, dr, 0)[0] / math.sqrt(4 * math.pi)
    rs = r[1:]
    exact = 1.0 / rs - (1.0 + 1.0 / rs) * np.exp(-2 * rs)
    return abs(V[0] - 1.0), np.max(np.abs(V[1:] - exact))


def test_hydrogen_1s():
    e0, e = _hydrogen_error(0.01)
    assert e0 < 1e-6 and e < 2e-6
    e0h, eh = _hydrogen_error(0.005)
    assert 7.0 < e0 / e0h < 9.0 and 7.0 < e / eh < 9.0


def test_l2_channel_against_quadrature():
    dr, Nr, l = 0.01, 3001, 2
    r = np.arange(Nr) * dr
    rho_lm = np.zeros((9, Nr))
    rho_lm[l * l + l] = r ** 2 * np.exp(-r)
    V = H.build_V_H(rho_lm, dr, 2)[l * l + l]
    R = r[-1]
    for k in (50, 200, 700, 2000):
        rk = r[k]
        inner = quad(lambda x: x ** 2 * math.exp(-x) * x ** (l + 2), 0, rk, epsabs=1e-14, epsrel=1e-13)[0]
        outer = quad(lambda x: x ** 2 * math.exp(-x) * x ** (1 - l), rk, R, epsabs=1e-14, epsrel=1e-13)[0]
        ref = 4 * math.pi / (2 * l + 1) * (inner / rk ** (l + 1) + rk ** l * outer)
        assert abs(V[k] - ref) <= 3e-6 * abs(ref)                # third order at dr = 0.01
    assert V[0] == 0.0


def test_guards():
    dr, Nr = 0.01, 10001                      # r up to 100: l above 690 / ln(100) = 149 is capped
    r = np.arange(Nr) * dr
    assert H.l_safe(r, 300) == min(int(690.0 / math.log(100.0)), 1 + int(690.0 / math.log(100.0)))
    rho = np.zeros((4, 201))
    rho[0] = np.exp(-np.arange(201) * 0.05)
    rho[2] = 1e-13                            # below the empty-channel threshold
    V = H.build_V_H(rho, 0.05, 1)
    assert np.all(V[1:] == 0.0) and np.all(np.isfinite(V[0]))

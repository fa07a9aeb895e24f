"""The oracle's K against exact phase shifts of a short-range well.

No reference test pins K to the physics.  Here a spherically symmetric
well U(r) = -exp(-(r/1.5)^2) enters through the L = 0 Hartree multipole
(V(mu, mu) gets V_H,00 / sqrt(4 pi)), with no nuclei and the one occupied
orbital scaled by 1e-8, so exchange is negligible.  Then K is diagonal and
K_ll follows from the phase shift delta_l of u'' = (l(l+1)/r^2 + 2U - k^2) u,
which scipy integrates to 1e-12 independently.

Two facts are checked.
- The sign convention: psi = J + Y K with Y = x y_l(x), and x y_0(x) =
  -cos x, so K = -tan(delta) in the convention u ~ sin(kr - l pi/2 + delta).
  The eigenphases atan(eig K) are therefore -delta.
- The grid: V(n) is taken at r = n dr while the recurrence runs on
  r = (n+1) dr.  K converges at first order in dr, and the Richardson
  value 2 K(dr/2) - K(dr) meets -tan(delta) to 1e-4.
"""
import math

import numpy as np
import pytest
from scipy.integrate import solve_ivp
from scipy.special import spherical_jn, spherical_yn

from oracle import solver as O
from scatt_b200.synth import ScanInputs

E = 0.5
L_CONT = 3


def U(r):
    return -np.exp(-(r / 1.5) ** 2)


def exact_delta(l, k, R):
    """delta_l from the radial equation integrated out to R (DOP853, rtol 1e-12)."""
    r0 = 1e-3
    sol = solve_ivp(lambda r, y: [y[1], (l * (l + 1) / r ** 2 + 2.0 * U(r) - k * k) * y[0]],
                    [r0, R], [r0 ** (l + 1), (l + 1) * r0 ** l], method="DOP853", rtol=1e-12, atol=1e-30)
    u, du = sol.y[0, -1], sol.y[1, -1]
    x = k * R
    j, dj = x * spherical_jn(l, x), k * (spherical_jn(l, x) + x * spherical_jn(l, x, derivative=True))
    n, dn = -x * spherical_yn(l, x), -k * (spherical_yn(l, x) + x * spherical_yn(l, x, derivative=True))
    return math.atan((u * dj - du * j) / (du * n - u * dn))     # u ~ j cos(delta) + n sin(delta)


def oracle_K(Nr, dr):
    r = np.arange(Nr) * dr
    F = np.zeros((1, 1, Nr))
    F[0, 0] = 1e-8 * 2.0 * np.exp(-r)
    VH = (math.sqrt(4.0 * math.pi) * U(r))[None, :]
    inp = ScanInputs(name="well", dr=dr, Nr=Nr, l_cont=L_CONT, atoms=np.zeros((0, 4)), psi_lm=F,
                     orb_energies=np.array([-0.5]), n_occ=1, V_H=VH)
    return O.solve_energy(O.make_setup(inp), E).K_kme


@pytest.fixture(scope="module")
def runs():
    return {dr: oracle_K(int(round(40.0 / dr)) + 1, dr) for dr in (0.01, 0.005)}


def test_K_is_diagonal_and_degenerate_in_m(runs):
    for K in runs.values():
        assert np.max(np.abs(K - np.diag(np.diag(K)))) <= 1e-12 * np.max(np.abs(K))
        for l in range(L_CONT + 1):
            block = np.diag(K)[l * l: (l + 1) * (l + 1)]
            assert np.max(block) - np.min(block) <= 1e-12 * max(abs(block[0]), 1e-300)


def test_K_meets_the_exact_phase_shifts(runs):
    k = math.sqrt(2.0 * E)
    K1, K2 = np.diag(runs[0.01]), np.diag(runs[0.005])
    for l in range(L_CONT + 1):
        mu = l * l + l
        target = -math.tan(exact_delta(l, k, 40.0))
        e1, e2 = K1[mu] - target, K2[mu] - target
        assert 1.8 < e1 / e2 < 2.2                                  # first order in dr
        assert abs(2.0 * K2[mu] - K1[mu] - target) < 2e-4           # Richardson
        assert abs(e2) < 0.02                                      # and close already at dr = 0.005


def test_dipole_phase_and_time_delay_follow_delta():
    """For one open channel D = conj((A - iB)^-1) d with d real, so arg D is
    +delta (the two sign choices above cancel) and the time delay of the
    default convention (oracle/observables.py, cross_section_delay.py) is the
    Wigner delay d delta / dE.  The s-like initial state reaches l = 1, m = 0
    in z only.  At dr = 0.005 both sit within the first-order grid error."""
    from oracle import observables as OBS
    dr, Nr = 0.005, 8001
    r = np.arange(Nr) * dr
    F = np.zeros((1, 1, Nr))
    F[0, 0] = 1e-8 * 2.0 * np.exp(-r)
    inp = ScanInputs(name="well", dr=dr, Nr=Nr, l_cont=2, atoms=np.zeros((0, 4)), psi_lm=F,
                     orb_energies=np.array([-0.5]), n_occ=1, V_H=(math.sqrt(4.0 * math.pi) * U(r))[None, :])
    st = O.make_setup(inp)
    Es = [0.49, 0.5, 0.51]
    res = [O.solve_energy(st, E_) for E_ in Es]
    k = [math.sqrt(2.0 * E_) for E_ in Es]
    mu = 2                                                    # l = 1, m = 0
    D = [list(x.slices[2]["D"]) for x in res]                 # (L, z)
    assert all(abs(d) <= 1e-12 * abs(row[mu]) for row in D for i, d in enumerate(row) if i != mu)
    delta = exact_delta(1, k[1], 40.0)
    assert abs(np.angle(D[1][mu]) - delta) < 0.01
    h = 1e-4
    ddelta_dE = (exact_delta(1, math.sqrt(2.0 * (Es[1] + h)), 40.0)
                 - exact_delta(1, math.sqrt(2.0 * (Es[1] - h)), 40.0)) / (2.0 * h)
    tau = OBS.time_delay(k, D)[1]
    assert ddelta_dE > 0 and abs(tau - ddelta_dE) < 0.03 * ddelta_dE

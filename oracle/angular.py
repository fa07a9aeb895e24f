"""Angular algebra of the oracle: (l, m) packing, Wigner 3j, real Gaunt.

Restates src/angular/Gaunt.hpp of the reference:
  * lm_to_idx / idx_to_lm ............ Gaunt.hpp:46-55
  * gaunt_complex_no_conj ............ Gaunt.hpp:65-87
  * U_real_to_complex ................ Gaunt.hpp:93-110
  * gaunt_real ....................... Gaunt.hpp:114-135
  * real_Ylm (+ sph_legendre_noCS) ... Gaunt.hpp:148-181
and the dipole helpers of src/scatt/DipoleMatrixElement.cpp:80-95.

The reference evaluates the 3j symbols with GSL (gsl_sf_coupling_3j, not
present in this image).  Here the 3j symbol is the Racah closed form summed
in exact rational arithmetic (Python integers), rounded once to double; it
is exact to the last bit, so it is at least as accurate as GSL's.
"""
from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

SQRT1_2 = math.sqrt(0.5)


def lm_to_idx(l: int, m: int) -> int:
    """Gaunt.hpp:46 -- idx = l*l + l + m."""
    return l * l + l + m


def idx_to_lm(idx: int) -> tuple[int, int]:
    """Gaunt.hpp:48-52."""
    l = int(math.sqrt(float(idx)))
    if (l + 1) * (l + 1) <= idx:
        l += 1
    return l, idx - l * l - l


@lru_cache(maxsize=None)
def _fact(n: int) -> int:
    return math.factorial(n)


@lru_cache(maxsize=1 << 20)
def wigner3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """Wigner 3j symbol for integer arguments (Racah formula, exact sum).

    Stands in for gsl_sf_coupling_3j(2j1, 2j2, 2j3, 2m1, 2m2, 2m3).
    """
    if m1 + m2 + m3 != 0:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    t1 = j2 - m1 - j3
    t2 = j1 + m2 - j3
    t3 = j1 + j2 - j3
    t4 = j1 - m1
    t5 = j2 + m2
    kmin = max(0, t1, t2)
    kmax = min(t3, t4, t5)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = (_fact(k) * _fact(k - t1) * _fact(k - t2) * _fact(t3 - k)
               * _fact(t4 - k) * _fact(t5 - k))
        s += Fraction(-1 if (k & 1) else 1, den)
    if s == 0:
        return 0.0
    tri = Fraction(_fact(j1 + j2 - j3) * _fact(j1 - j2 + j3) * _fact(-j1 + j2 + j3),
                   _fact(j1 + j2 + j3 + 1))
    pre = (_fact(j1 + m1) * _fact(j1 - m1) * _fact(j2 + m2) * _fact(j2 - m2)
           * _fact(j3 + m3) * _fact(j3 - m3))
    sq = tri * pre * s * s
    sign = -1.0 if ((j1 - j2 - m3) & 1) else 1.0
    if s < 0:
        sign = -sign
    return sign * math.sqrt(float(sq))


def gaunt_complex_no_conj(l1, m1, l2, m2, l3, m3) -> float:
    """Gaunt.hpp:65-87 -- integral Y_l1m1 Y_l2m2 Y_l3m3 (no conjugation)."""
    if m1 + m2 + m3 != 0:
        return 0.0
    if abs(l1 - l2) > l3:
        return 0.0
    if l1 + l2 < l3:
        return 0.0
    if (l1 + l2 + l3) & 1:
        return 0.0
    w000 = wigner3j(l1, l2, l3, 0, 0, 0)
    wmmm = wigner3j(l1, l2, l3, m1, m2, m3)
    pre = math.sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0) * (2.0 * l3 + 1.0) / (4.0 * math.pi))
    return pre * w000 * wmmm


def _phase(m: int) -> float:
    return -1.0 if (m & 1) else 1.0


def U_real_to_complex(mR: int, mC: int) -> complex:
    """Gaunt.hpp:93-110 -- Y^complex_mC = sum_mR U Y^real_mR coefficient."""
    if mR == 0:
        return 1.0 + 0j if mC == 0 else 0j
    if mR > 0:
        if mC == -mR:
            return complex(SQRT1_2, 0.0)
        if mC == mR:
            return complex(SQRT1_2 * _phase(mR), 0.0)
        return 0j
    p = -mR
    if mC == -p:
        return complex(0.0, SQRT1_2)
    if mC == p:
        return complex(0.0, -SQRT1_2 * _phase(p))
    return 0j


def m3_candidates(m1: int, m2: int, l3: int):
    """Real-harmonic m3 with a possibly nonzero real Gaunt coefficient for
    (m1, m2): |m3| = |m1| + |m2| or ||m1| - |m2||; every other m3 gives exactly 0
    (no complex m-triple sums to zero).  Ascending, within |m3| <= l3."""
    a, b = abs(m1), abs(m2)
    mags = {a + b, abs(a - b)}
    out = set()
    for x in mags:
        if x <= l3:
            out.add(x)
            out.add(-x)
    return sorted(out)


def _m_candidates(mR: int):
    """Complex m values with U_real_to_complex(mR, m) != 0, ascending."""
    a = abs(mR)
    return (0,) if a == 0 else (-a, a)


@lru_cache(maxsize=1 << 22)
def gaunt_real(l1, mR1, l2, mR2, l3, mR3) -> float:
    """Gaunt.hpp:114-135 -- integral of three real spherical harmonics.

    The reference sums over every (m1, m2) with m3 = -(m1 + m2); only
    m = +-|mR| carry a nonzero U coefficient, so the loops visit exactly those
    (in the same ascending order, hence the same accumulation order)."""
    if abs(l1 - l2) > l3 or l1 + l2 < l3:
        return 0.0
    if (l1 + l2 + l3) & 1:
        return 0.0
    acc = 0j
    for m1 in _m_candidates(mR1):
        if m1 < -l1 or m1 > l1:
            continue
        U1 = U_real_to_complex(mR1, m1)
        if U1 == 0:
            continue
        for m2 in _m_candidates(mR2):
            if m2 < -l2 or m2 > l2:
                continue
            U2 = U_real_to_complex(mR2, m2)
            if U2 == 0:
                continue
            m3 = -(m1 + m2)
            if m3 < -l3 or m3 > l3:
                continue
            U3 = U_real_to_complex(mR3, m3)
            if U3 == 0:
                continue
            Gc = gaunt_complex_no_conj(l1, m1, l2, m2, l3, m3)
            if Gc == 0.0:
                continue
            acc += U1 * U2 * U3 * Gc
    return acc.real


def sph_legendre_noCS(l: int, m: int, theta: float) -> float:
    """Gaunt.hpp:148-168 -- orthonormal associated Legendre, no Condon-Shortley."""
    if l < 0 or m < 0 or m > l:
        return 0.0
    s, c = math.sin(theta), math.cos(theta)
    S_mm = 1.0 / math.sqrt(4.0 * math.pi)
    for k in range(1, m + 1):
        S_mm *= math.sqrt((2.0 * k + 1.0) / (2.0 * k)) * s
    if l == m:
        return S_mm
    S_prev = S_mm
    S_cur = math.sqrt(2.0 * m + 3.0) * c * S_mm
    if l == m + 1:
        return S_cur
    S_pp = S_prev
    S_prev = S_cur
    for k in range(m + 2, l + 1):
        a = math.sqrt((4.0 * k * k - 1.0) / (float(k) * k - m * m))
        b = math.sqrt((float(k - 1) * (k - 1) - m * m) / (4.0 * (k - 1.0) * (k - 1.0) - 1.0))
        S_k = a * (c * S_prev - b * S_pp)
        S_pp = S_prev
        S_prev = S_k
    return S_prev


def real_Ylm(l: int, m: int, theta: float, phi: float) -> float:
    """Gaunt.hpp:171-181."""
    if l < 0 or abs(m) > l:
        return 0.0
    am = abs(m)
    S = sph_legendre_noCS(l, am, theta)
    if m == 0:
        return S
    if m > 0:
        return math.sqrt(2.0) * S * math.cos(m * phi)
    return math.sqrt(2.0) * S * math.sin(am * phi)


def angular_dipole(l_mu, m_mu, q, l_nu, m_nu) -> float:
    """DipoleMatrixElement.cpp:80-88 -- sqrt(4pi/3) * G^R(l_mu m_mu; 1 q; l_nu m_nu)."""
    return math.sqrt(4.0 * math.pi / 3.0) * gaunt_real(l_mu, m_mu, 1, q, l_nu, m_nu)


def velocity_coef(l_mu, l_nu) -> float:
    """DipoleMatrixElement.cpp:90-95."""
    if l_mu == l_nu + 1:
        return -float(l_nu + 1)
    if l_mu == l_nu - 1:
        return float(l_nu)
    return 0.0


def build_G_vector(n_mu: int, n_lambda: int, n_sigma: int):
    """WavefunctionSetup.cpp:21-81 -- non-zero G^R_{mu,lambda,sigma} (|G| > 1e-14).

    Enumerates only the (l, m) combinations the selection rules allow
    (triangle, parity, |m_sigma| = |m_mu| +- |m_lambda|); the values and the
    1e-14 cut are the reference's.
    Returns a list of (mu, lambda, sigma, value) sorted by (mu, lambda, sigma).
    """
    lmax_mu = idx_to_lm(n_mu - 1)[0]
    lmax_la = idx_to_lm(n_lambda - 1)[0]
    lmax_si = idx_to_lm(n_sigma - 1)[0]
    out = []
    for mu in range(n_mu):
        lm, mm = idx_to_lm(mu)
        for ll in range(0, lmax_la + 1):
            for ls in range(abs(lm - ll), min(lm + ll, lmax_si) + 1):
                if (lm + ll + ls) & 1:
                    continue
                for ml in range(-ll, ll + 1):
                    la = lm_to_idx(ll, ml)
                    if la >= n_lambda:
                        continue
                    for ms in m3_candidates(mm, ml, ls):
                        si = lm_to_idx(ls, ms)
                        if si >= n_sigma:
                            continue
                        v = gaunt_real(lm, mm, ll, ml, ls, ms)
                        if abs(v) > 1e-14:
                            out.append((mu, la, si, v))
    out.sort(key=lambda t: (t[0], t[1], t[2]))
    return out

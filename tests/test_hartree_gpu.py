"""The device Hartree step of preprocessing (scatt_hartree: the radial
Poisson integrals of preprocessing/src/potential/Hartree.hpp:71-246) against
the oracle's restatement (oracle/hartree.py, itself held to the hydrogen 1s
potential and to quadrature in tests/test_oracle_hartree.py).  Same
integrator, same guards; the prefix sums run in a different order (a
block-wide scan against a sequential cumsum).

Tolerance: 1e-12 of the channel's largest value plus the summation floor
of the reference's formula.  The outer term is r^l (I_out(R) - I_out(r)),
a difference of two running sums times r^l, so at large r and l any two
summation orders differ by up to the recursive-summation bound
(n - 1) eps sum |increments| of each sum, times r^l -- about 1e-9 of the
channel's scale at l = 6, r = 25 (the oracle's own cumsum is no closer to
the exact value than that).  The floor adds those bounds point by point,
and the inner term's k eps sum_{j<k} |increment| / r^(l+1)."""
import math

import numpy as np
import pytest

from oracle import hartree as H
from scatt_b200 import _lib

pytestmark = pytest.mark.gpu


def _density(l_max, Nr, dr, r0=0.0, seed=3):
    """Smooth multipoles rho_lm ~ r^l exp(-a r) with seeded amplitudes; the
    odd-m channels of l = 3 are left below the 1e-12 threshold."""
    rng = np.random.default_rng(seed)
    r = r0 + np.arange(Nr) * dr
    rho = np.zeros(((l_max + 1) ** 2, Nr))
    for ch in range(rho.shape[0]):
        l = math.isqrt(ch)
        m = ch - l * l - l
        amp = rng.standard_normal() * (1e-14 if (l == 3 and m % 2) else 1.0)
        rho[ch] = amp * r ** l * np.exp(-(0.9 + 0.1 * l) * r)
    return rho


def summation_floor(rho, dr, l_max, r0=0.0):
    """Point-wise bound on how far two summation orders of the reference's
    running integrals can move V_lm: 2 (n - 1) eps S_out r^l + 2 k eps
    (C_out(k) r^l + C_in(k) / r^(l+1)), with S the sum and C(k) the prefix
    sum of the increments' magnitudes (14/12 dr |f| bounds an increment's)."""
    eps = np.finfo(np.float64).eps
    Nr = rho.shape[1]
    r = r0 + np.arange(Nr) * dr
    k = np.arange(Nr)
    out = np.zeros(((l_max + 1) ** 2, Nr))
    with np.errstate(all="ignore"):
        for ch in range(out.shape[0]):
            l = math.isqrt(ch)
            pref = 4.0 * math.pi / (2.0 * l + 1.0)
            a = np.abs(rho[ch]) * r ** (l + 2)
            b = np.abs(rho[ch]) * (r if l == 0 else np.where(r <= 0.0, 0.0, np.where(r <= 0.0, 1.0, r) ** (1 - l)))
            ca = np.concatenate([[0.0], np.cumsum(a[:-1])]) * (14.0 / 12.0) * dr
            cb = np.concatenate([[0.0], np.cumsum(b[:-1])]) * (14.0 / 12.0) * dr
            sb = np.sum(b) * (14.0 / 12.0) * dr
            inner = np.where(r <= 0.0, 0.0, 2.0 * k * eps * ca / np.where(r <= 0.0, 1.0, r) ** (l + 1))
            outer = 2.0 * ((Nr - 1) * eps * sb + k * eps * cb) * r ** l
            f = pref * (inner + outer)
            out[ch] = np.where(np.isfinite(f), f, np.inf)
    return out


@pytest.mark.parametrize("Nr,dr,r0", [(2001, 0.01, 0.0), (1500, 0.02, 0.05), (3, 0.1, 0.0)])
def test_hartree_matches_oracle(Nr, dr, r0):
    l_max = 6
    rho = _density(l_max, Nr, dr, r0)
    got = _lib.hartree(rho, dr, l_max, r0)
    ref = H.build_V_H(rho, dr, l_max, r0)
    assert got.shape == ref.shape
    fl = summation_floor(rho, dr, l_max, r0)
    for ch in range(ref.shape[0]):
        scale = max(np.max(np.abs(ref[ch])), 1e-300)
        assert np.all(np.abs(got[ch] - ref[ch]) <= 1e-12 * scale + fl[ch]), ch
    for ch in (9, 11, 13, 15):                     # l = 3, odd m: below the 1e-12 threshold
        assert np.all(got[ch] == 0.0) and np.all(ref[ch] == 0.0)


def test_hartree_overflow_cap_and_extra_rows():
    """A grid starting at r0 = 1e-100 caps l at 1 + 690 / ln(1e100) = 3:
    channels with l > 3 stay 0, as in the reference; rows beyond
    (l_max + 1)^2 are ignored."""
    l_max, Nr, dr, r0 = 5, 400, 0.05, 1e-100
    rho = np.vstack([_density(l_max, Nr, dr, r0), np.ones((3, Nr))])
    got = _lib.hartree(rho, dr, l_max, r0)
    ref = H.build_V_H(rho, dr, l_max, r0)
    assert H.l_safe(r0 + np.arange(Nr) * dr, l_max) == 3
    assert np.all(got[16:] == 0.0)
    fl = summation_floor(rho[:36], dr, l_max, r0)
    for ch in range(16):
        scale = max(np.max(np.abs(ref[ch])), 1e-300)
        assert np.all(np.abs(got[ch] - ref[ch]) <= 1e-12 * scale + fl[ch]), ch


def test_hartree_rejects_short_rows():
    with pytest.raises(_lib.ScattError):
        _lib.hartree(np.zeros((3, 50)), 0.1, 1)

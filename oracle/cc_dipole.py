"""Continuum-continuum dipole between two scattering states.  TEST
INFRASTRUCTURE ONLY (the oracle for a device version of this consumer).

Restates postprocessing/two_photon_delay/cc_dipole/src/CCDipole.cpp, the
consumer of the back-propagated psi that the two-photon delay analysis
runs after the scattering pipeline:

    cc_raw[beta, alpha] = sum_ir w_ir r_ir psi_kappa(ir)[:, beta]^T A^q psi_nu(ir)[:, alpha]

in the back-propagation basis, length gauge only (CCDipole.cpp:294-303
rejects the velocity gauge), with r = r_min + ir dr (r_min = dr,
CCDipole.cpp:236), A^q_{mu nu} = sqrt(4 pi / 3) gaunt_real(l_mu, m_mu, 1, q,
l_nu, m_nu) (:135-160), q = +1 / -1 / 0 for x / y / z, Simpson weights of
:100-122 over the overlap of the two kept windows (:79-95).
"""
from __future__ import annotations

import numpy as np

from . import angular

Q_OF = {"x": 1, "y": -1, "z": 0}


def window(n_grid, keep_kappa, keep_nu, n_overlap_hi=-1):
    """CCDipole.cpp:79-95 -- [n_lo, n_hi) from the two (n_keep_lo, n_keep_hi) ranges."""
    n_lo = max(0, keep_kappa[0], keep_nu[0])
    n_hi = min(n_grid, keep_kappa[1] + 1, keep_nu[1] + 1)
    if n_overlap_hi > 0:
        n_hi = min(n_hi, n_overlap_hi)
    if n_hi - n_lo < 5:
        raise RuntimeError(f"cc_dipole: too few overlapping radial points (n_lo={n_lo}, n_hi={n_hi})")
    return n_lo, n_hi


def simpson_weights(n_pts, h):
    """CCDipole.cpp:100-122."""
    w = np.zeros(n_pts)
    if n_pts % 2 == 1:
        w[0] = w[n_pts - 1] = h / 3.0
        for i in range(1, n_pts - 1):
            w[i] = (4.0 if i & 1 else 2.0) * h / 3.0
        return w
    n13 = n_pts - 3
    if n13 >= 2:
        w[0] += h / 3.0
        w[n13 - 1] += h / 3.0
        for i in range(1, n13 - 1):
            w[i] += (4.0 if i & 1 else 2.0) * h / 3.0
    s38 = 3.0 * h / 8.0
    j = n_pts - 4
    w[j] += s38
    w[j + 1] += 3.0 * s38
    w[j + 2] += 3.0 * s38
    w[j + 3] += s38
    return w


def ang_table(n_mu, q):
    """CCDipole.cpp:135-160 as a dense table."""
    lm = [angular.idx_to_lm(mu) for mu in range(n_mu)]
    A = np.zeros((n_mu, n_mu))
    for mu, (l1, m1) in enumerate(lm):
        for nu, (l2, m2) in enumerate(lm):
            if abs(l1 - l2) == 1:
                A[mu, nu] = angular.angular_dipole(l1, m1, q, l2, m2)
    return A


def cc_dipole(dr, n_grid, psi_kappa, psi_nu, keep_kappa, keep_nu, pol, gauge="length", n_overlap_hi=-1):
    """CCDipole.cpp:294-334: cc_raw (N_psi x N_psi) of one (kappa, nu) pair.
    psi_*: {ir: (N_psi, N_psi) array}; keep_*: (n_keep_lo, n_keep_hi)."""
    if gauge != "length":
        raise RuntimeError("compute_cc_dipole: only length gauge implemented in this pass")
    n_lo, n_hi = window(n_grid, keep_kappa, keep_nu, n_overlap_hi)
    n_mu = next(iter(psi_kappa.values())).shape[0]
    A = ang_table(n_mu, Q_OF[pol])
    w = simpson_weights(n_hi - n_lo, dr)
    cc = np.zeros((n_mu, n_mu))
    for ir in range(n_lo, n_hi):
        r = dr + ir * dr
        cc += (w[ir - n_lo] * r) * (psi_kappa[ir].T @ (A @ psi_nu[ir]))
    return cc

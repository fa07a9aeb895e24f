"""Single-centre expansion of a function sampled on the preprocessing's
angular grid.  TEST INFRASTRUCTURE ONLY (the oracle for the device
projection, scatt_sce_project).

Restates preprocessing/src/sce/SCE.hpp:122-266 (project, direct-DFT
backend) on the grid of preprocessing/src/angular/Grid.hpp:
n_theta = Lmax + 1 Gauss-Legendre nodes x_i = cos(theta_i) in ascending
order (GaussLegendre.hpp), n_phi = 2 (Lmax + 1) nodes phi_j = 2 pi j / n_phi:

    A_m(theta_i) = sum_j F(theta_i, phi_j) cos(m phi_j),  B_m = sum_j F sin(m phi_j)
    F_{l,0}   = dphi sum_i w_i S_{l,0}(theta_i) A_0(theta_i)
    F_{l,+m}  = sqrt(2) dphi sum_i w_i S_{l,m}(theta_i) A_m(theta_i)
    F_{l,-m}  = sqrt(2) dphi sum_i w_i S_{l,m}(theta_i) B_m(theta_i)

with dphi = 2 pi / n_phi and S_{l,m} the normalised associated Legendre
function without the Condon-Shortley phase (angular/Legendre.hpp:11-31,
sph_legendre_noCS), by the standard recurrence of Holmes and Featherstone
(2002) that the reference uses.
"""
from __future__ import annotations

import math

import numpy as np


def grid(Lmax: int):
    """(cos_theta, weights, theta, phi) of the angular grid for Lmax."""
    x, w = np.polynomial.legendre.leggauss(Lmax + 1)          # ascending
    n_phi = 2 * (Lmax + 1)
    phi = 2.0 * math.pi * np.arange(n_phi) / n_phi
    return x, w, np.arccos(x), phi


def s_table(Lmax: int, theta: np.ndarray) -> np.ndarray:
    """S[l, m, i] = S_{l,m}(theta_i) for 0 <= m <= l <= Lmax (0 above)."""
    s, c = np.sin(theta), np.cos(theta)
    S = np.zeros((Lmax + 1, Lmax + 1, theta.size))
    smm = np.full(theta.size, 1.0 / math.sqrt(4.0 * math.pi))
    for m in range(Lmax + 1):
        if m > 0:
            smm = smm * math.sqrt((2.0 * m + 1.0) / (2.0 * m)) * s
        S[m, m] = smm
        if m + 1 <= Lmax:
            S[m + 1, m] = math.sqrt(2.0 * m + 3.0) * c * smm
        for k in range(m + 2, Lmax + 1):
            a = math.sqrt((4.0 * k * k - 1.0) / (k * k - m * m))
            b = math.sqrt(((k - 1) ** 2 - m * m) / (4.0 * (k - 1) ** 2 - 1.0))
            S[k, m] = a * (c * S[k - 1, m] - b * S[k - 2, m])
    return S


def real_ylm(l: int, m: int, theta, phi):
    """Y^R_{l,m} of the grid's convention (SCE.hpp:11-15)."""
    S = s_table(l, np.atleast_1d(theta))[l, abs(m)]
    if m == 0:
        return S
    if m > 0:
        return math.sqrt(2.0) * S * np.cos(m * phi)
    return math.sqrt(2.0) * S * np.sin(-m * phi)


def project(samples: np.ndarray, Lmax: int) -> np.ndarray:
    """SCE.hpp:122-266: F_lm (Nlm, Nr) from samples (Nr, n_theta, n_phi),
    samples[k, i, j] = F(r_k, theta_i, phi_j)."""
    x, w, theta, phi = grid(Lmax)
    n_t, n_p = x.size, phi.size
    Nr = samples.shape[0]
    assert samples.shape == (Nr, n_t, n_p)
    S = s_table(Lmax, theta)
    dphi = 2.0 * math.pi / n_p
    m = np.arange(Lmax + 1)
    cosM = np.cos(np.outer(m, phi))                     # (Lmax + 1, n_phi)
    sinM = np.sin(np.outer(m, phi))
    A = np.einsum("kij,mj->kmi", samples, cosM)        # (Nr, Lmax + 1, n_theta)
    B = np.einsum("kij,mj->kmi", samples, sinM)
    out = np.zeros(((Lmax + 1) ** 2, Nr))
    for l in range(Lmax + 1):
        out[l * l + l] = dphi * np.einsum("i,i,ki->k", w, S[l, 0], A[:, 0])
        for mm in range(1, l + 1):
            ws = w * S[l, mm]
            out[l * l + l + mm] = math.sqrt(2.0) * dphi * (A[:, mm] @ ws)
            out[l * l + l - mm] = math.sqrt(2.0) * dphi * (B[:, mm] @ ws)
    return out


def synthesize(coef: np.ndarray, Lmax: int) -> np.ndarray:
    """Samples (Nr, n_theta, n_phi) of F = sum_lm coef[lm, k] Y^R_lm on the
    grid of Lmax (coef may hold fewer channels than (Lmax + 1)^2)."""
    _, _, theta, phi = grid(Lmax)
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    out = np.zeros((coef.shape[1], theta.size, phi.size))
    for ch in range(coef.shape[0]):
        l = math.isqrt(ch)
        m = ch - l * l - l
        Y = np.stack([real_ylm(l, m, TH[i], PH[i]) for i in range(theta.size)])
        out += coef[ch][:, None, None] * Y[None]
    return out


def synthesize_at(F_lm: np.ndarray, r0: float, dr: float, origin, Lmax: int, P) -> float:
    """preprocessing/src/sce/Synthesize.hpp:23-97: F(P) = sum_lm F_lm(r) Y^R_lm
    at the point P, F_lm (>= (Lmax + 1)^2 rows, Nr columns) on r_k = r0 + k dr,
    by 4-point Lagrange interpolation in r on the stencil k - 1 .. k + 2
    (k = floor((r - r0) / dr) clamped to 1 .. Nr - 3); 0 outside the grid."""
    d = np.asarray(P, dtype=np.float64) - np.asarray(origin, dtype=np.float64)
    r = float(np.sqrt(d @ d))
    Nr = F_lm.shape[1]
    if r < r0 - 1e-14 or r > r0 + (Nr - 1) * dr + 1e-14:
        return 0.0
    theta = phi = 0.0
    if r > 1e-14:
        theta = math.acos(min(1.0, max(-1.0, d[2] / r)))
        phi = math.atan2(d[1], d[0])
    k = min(max(int(math.floor((r - r0) / dr)), 1), Nr - 3)
    s = (r - (r0 + k * dr)) / dr
    w = np.array([-s * (s - 1.0) * (s - 2.0) / 6.0, (s + 1.0) * (s - 1.0) * (s - 2.0) * 0.5,
                  -(s + 1.0) * s * (s - 2.0) * 0.5, (s + 1.0) * s * (s - 1.0) / 6.0])
    n_lm = (Lmax + 1) ** 2
    Fr = F_lm[:n_lm, k - 1:k + 3] @ w
    S = s_table(Lmax, np.array([theta]))[:, :, 0]
    out = 0.0
    for l in range(Lmax + 1):
        out += Fr[l * l + l] * S[l, 0]
        for m in range(1, l + 1):
            out += Fr[l * l + l + m] * math.sqrt(2.0) * S[l, m] * math.cos(m * phi)
            out += Fr[l * l + l - m] * math.sqrt(2.0) * S[l, m] * math.sin(m * phi)
    return float(out)

"""Contracted spherical-Gaussian basis, its molecular orbitals and density,
sampled on the single-centre expansion's grid.  TEST INFRASTRUCTURE ONLY
(the oracle for scatt_sce_basis).

Restates preprocessing/src/basis/MoldenBasis.hpp:48-229 (AtomicOrbital::eval,
molden_index_to_m, build_basis, evaluate_mo, evaluate_density),
SphericalGaussian.hpp / Primitive.hpp (the normalisation) and
potential/LocalExchange.hpp (the local exchange of the density):

    chi_lm(r) = |r - A|^l Y^R_lm(r - A) sum_a c~_a exp(-alpha_a |r - A|^2)
    c~_a = s c_a N_sph(alpha_a, l),  N_sph^2 = 2^(2l + 7/2) alpha^(l + 3/2) / (sqrt(pi) (2l + 1)!!)
    s = 1 / sqrt(sum_ab c_a c_b (2 sqrt(alpha_a alpha_b) / (alpha_a + alpha_b))^(l + 3/2))

with the AOs of a shell in molden order (p: m = +1, -1, 0; l >= 2:
m = 0, +1, -1, +2, -2, ...), psi_i = sum_mu C_i,mu chi_mu and
rho = sum_i n_i psi_i^2.  Y^R_lm is oracle.sce.real_ylm (no Condon-Shortley
phase).  A shell is (center (3,), l, exponents, coefficients).
"""
from __future__ import annotations

import math

import numpy as np

from . import sce as SC


def molden_m(l: int, idx: int) -> int:
    """MoldenBasis.hpp:110-127."""
    if l == 0:
        return 0
    if l == 1:
        return (1, -1, 0)[idx]
    if idx == 0:
        return 0
    half = (idx + 1) // 2
    return half if idx & 1 else -half


def n_sph(alpha: float, l: int) -> float:
    dfact = 1.0
    for k in range(1, l + 1):
        dfact *= 2.0 * k + 1.0
    return math.sqrt(2.0 ** (2.0 * l + 3.5) * alpha ** (l + 1.5) / (math.sqrt(math.pi) * dfact))


def c_tilde(l: int, exps, coefs) -> np.ndarray:
    exps = np.asarray(exps, dtype=np.float64)
    coefs = np.asarray(coefs, dtype=np.float64)
    p = 2.0 * np.sqrt(np.outer(exps, exps)) / (exps[:, None] + exps[None, :])
    so = float(coefs @ (p ** (l + 1.5)) @ coefs)
    return coefs / math.sqrt(so) * np.array([n_sph(a, l) for a in exps])


def ao_values(shells, pts: np.ndarray) -> np.ndarray:
    """(nbf, n_points): every AO at absolute positions pts (n, 3)."""
    rows = []
    for center, l, exps, coefs in shells:
        d = pts - np.asarray(center)[None, :]
        r2 = np.sum(d * d, axis=1)
        r = np.sqrt(r2)
        ct = c_tilde(l, exps, coefs)
        rad = np.exp(-np.outer(r2, exps)) @ ct
        safe = r > 1e-300
        theta = np.arccos(np.clip(np.where(safe, d[:, 2] / np.where(safe, r, 1.0), 1.0), -1.0, 1.0))
        phi = np.arctan2(d[:, 1], d[:, 0])
        for idx in range(1 if l == 0 else 2 * l + 1):
            m = molden_m(l, idx)
            y = SC.real_ylm(l, m, theta, phi) * (r ** l if l else 1.0)
            y = np.where(safe, y, (1.0 / math.sqrt(4.0 * math.pi)) if l == 0 else 0.0)
            rows.append(y * rad)
    return np.array(rows)


def grid_points(Lmax: int, radii: np.ndarray, origin) -> np.ndarray:
    """(Nr n_theta n_phi, 3): origin + r (sin t cos p, sin t sin p, cos t), order [r][theta][phi]."""
    x, _, theta, phi = SC.grid(Lmax)
    st = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    dirs = np.stack([np.outer(st, np.cos(phi)), np.outer(st, np.sin(phi)),
                     np.outer(x, np.ones_like(phi))], axis=-1).reshape(-1, 3)
    return (np.asarray(origin)[None, None, :] + radii[:, None, None] * dirs[None]).reshape(-1, 3)


def v_x_local(rho: np.ndarray, form: int) -> np.ndarray:
    """LocalExchange.hpp:28-47: -(3/pi)^(1/3) rho^(1/3) (form 1, Slater) or
    1.5 times that (form 2, Kohn-Sham), rho clamped at 0."""
    c = (3.0 / math.pi) ** (1.0 / 3.0) * (1.0 if form == 1 else 1.5)
    return -c * np.cbrt(np.maximum(0.0, rho))


def sce_of_basis(shells, C, occ, Lmax: int, radii: np.ndarray, origin, vx_form: int = 0):
    """(orb_lm (n_mo, Nlm, Nr), rho_lm (Nlm, Nr)), with vx_lm (Nlm, Nr) when
    vx_form is 1 or 2: the SCE projections (oracle.sce.project) of every MO,
    of the density and of the local exchange."""
    pts = grid_points(Lmax, radii, origin)
    chi = ao_values(shells, pts)                               # (nbf, P)
    psi = np.asarray(C) @ chi                                  # (n_mo, P)
    rho = np.asarray(occ) @ (psi * psi)
    shape = (radii.size, Lmax + 1, 2 * (Lmax + 1))
    orb = np.stack([SC.project(psi[i].reshape(shape), Lmax) for i in range(psi.shape[0])])
    rho_lm = SC.project(rho.reshape(shape), Lmax)
    if vx_form:
        return orb, rho_lm, SC.project(v_x_local(rho, vx_form).reshape(shape), Lmax)
    return orb, rho_lm

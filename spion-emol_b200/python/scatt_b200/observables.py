"""Photoionisation observables of a scan: cross sections and Wigner time delays.

These are the quantities the reference derives from the dipoles it writes
(postprocessing/cross_section_delay.py:195-263; constants :120-122), here
computed on the host from the solver's outputs for a whole energy grid:

    sigma_L(omega) = 8 pi omega / (c k) * sum_mu |D^L_mu|^2
    sigma_V(omega) = 8 pi / (c k omega) * sum_mu |D^V_mu|^2
    tau(E)         = Im[ sum_mu conj(D_mu) dD_mu/dE ] / sum_mu |D_mu|^2
    q              = sum |D^V|^2 / (omega^2 sum |D^L|^2)

with dD/dE = (dD/dk) / k, dD/dk by second-order finite differences on the
(possibly uneven) k grid (one-sided at the ends), and omega = E - E_HOMO
(src/scatt/DipoleIO.cpp:285).  D is the orthogonalised reduced dipole
(DipoleResult::D_reduced) of one slot; the six slots are (L,x) (L,y) (L,z)
(V,x) (V,y) (V,z).  Also, as cross_section_delay.py:270-430 computes them:

    dphi_rms = sqrt( sum w dphi^2 / sum w ),  dphi = arg(D^V conj D^L),  w = |D^L| |D^V|
    beta     = N_1 / sigma_tot - 1   (orientation-averaged asymmetry, linear polarisation)
    sigma_tot = 1/3 int dOmega sum_q |D^(q)(k)|^2,   N_1 = int dOmega |sum_q D^(q)(k) k_q|^2,
    D^(q)(k) = sum_lm d^(q)_lm Y^R_lm(k)

with the integrals on a Gauss-Legendre (cos theta) x trapezoid (phi) grid,
40 x 80 by default, which is exact while 2 (l_max + 1) < 80.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import sph_harm_y

C_AU = 137.036            # speed of light, atomic units
AU_TO_AS = 24.18884       # atomic unit of time in attoseconds
SLOTS = [("length", "x"), ("length", "y"), ("length", "z"),
         ("velocity", "x"), ("velocity", "y"), ("velocity", "z")]


def cross_section(k, D, omega, gauge: str) -> np.ndarray:
    """Total cross section in bohr^2 per energy; D has shape (n_energy, n_channels)."""
    k = np.asarray(k, dtype=np.float64)
    omega = np.asarray(omega, dtype=np.float64)
    s2 = np.sum(np.abs(np.asarray(D)) ** 2, axis=1)
    if gauge == "length":
        return 8.0 * np.pi * omega / (C_AU * k) * s2
    if gauge == "velocity":
        return 8.0 * np.pi / (C_AU * k * omega) * s2
    raise ValueError(f"unknown gauge {gauge!r}")


def time_delay(k, D, with_minus: bool = False) -> np.ndarray:
    """Wigner delay in atomic time units per energy (D: (n_energy, n_channels)).

    with_minus flips the sign (the reference's opt-in legacy convention)."""
    k = np.asarray(k, dtype=np.float64)
    D = np.asarray(D, dtype=np.complex128)
    if k.size < 2:
        raise ValueError("the time delay needs at least two energies")
    dD_dE = np.gradient(D, k, axis=0) / k[:, None]
    num = np.sum(np.conj(D) * dD_dE, axis=1).imag
    den = np.sum(np.abs(D) ** 2, axis=1)
    tau = np.divide(num, den, out=np.zeros_like(num), where=den > 1e-30)
    return -tau if with_minus else tau


def q_sigma(D_L, D_V, omega) -> np.ndarray:
    """Gauge-consistency ratio sum|D_V|^2 / (omega^2 sum|D_L|^2) (1 for exact states)."""
    omega = np.asarray(omega, dtype=np.float64)
    den = omega ** 2 * np.sum(np.abs(np.asarray(D_L)) ** 2, axis=1)
    num = np.sum(np.abs(np.asarray(D_V)) ** 2, axis=1)
    return np.divide(num, den, out=np.full_like(num, np.nan), where=den > 1e-30)


def dphi_rms(D_L, D_V) -> np.ndarray:
    """Weighted rms phase difference between the gauges, per energy
    (cross_section_delay.py:270-275); D_L, D_V: (n_energy, n_channels)."""
    D_L = np.asarray(D_L, dtype=np.complex128)
    D_V = np.asarray(D_V, dtype=np.complex128)
    dphi = np.angle(D_V * np.conj(D_L))
    w = np.abs(D_L) * np.abs(D_V)
    s_w = np.sum(w, axis=1)
    s_w_phi2 = np.sum(w * dphi ** 2, axis=1)
    return np.sqrt(np.divide(s_w_phi2, s_w, out=np.zeros_like(s_w_phi2), where=s_w > 1e-30))


def real_ylm(l: int, m: int, theta, phi):
    """Real spherical harmonic without the Condon-Shortley phase
    (src/angular/Gaunt.hpp:171-181): x <-> m = +1, y <-> m = -1, z <-> m = 0."""
    am = abs(m)
    if m == 0:
        return np.real(sph_harm_y(l, 0, theta, phi))
    if m > 0:
        return math.sqrt(2.0) * (-1.0) ** m * np.real(sph_harm_y(l, m, theta, phi))
    return math.sqrt(2.0) * (-1.0) ** am * np.imag(sph_harm_y(l, am, theta, phi))


def beta(D_x, D_y, D_z, mu_list=None, n_theta: int = 40, n_phi: int = 80) -> np.ndarray:
    """Orientation-averaged asymmetry parameter per energy, in [-1, 2]
    (cross_section_delay.py:350-430).  D_q: (n_energy, n_channels) dipoles of
    the three polarisations; mu_list: the lm index of each channel (default
    0 .. n_channels - 1)."""
    D = [np.asarray(d, dtype=np.complex128) for d in (D_x, D_y, D_z)]
    n_ch = D[0].shape[1]
    mu_list = list(range(n_ch)) if mu_list is None else list(mu_list)
    x, w = np.polynomial.legendre.leggauss(n_theta)
    theta = np.arccos(x)
    phi = np.arange(n_phi) * (2.0 * np.pi / n_phi)
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    Y = np.empty((n_ch, n_theta, n_phi))
    for i, mu in enumerate(mu_list):
        l = int(math.isqrt(mu))
        Y[i] = real_ylm(l, mu - l * l - l, TH, PH)
    weights = w[:, None] * (2.0 * np.pi / n_phi)
    maps = [np.tensordot(d, Y, axes=([1], [0])) for d in D]          # (n_energy, n_theta, n_phi)
    sigma_tot = np.sum((np.abs(maps[0]) ** 2 + np.abs(maps[1]) ** 2 + np.abs(maps[2]) ** 2)
                       * weights, axis=(1, 2)) / 3.0
    k_dot = maps[0] * (np.sin(TH) * np.cos(PH)) + maps[1] * (np.sin(TH) * np.sin(PH)) + maps[2] * np.cos(TH)
    N1 = np.sum(np.abs(k_dot) ** 2 * weights, axis=(1, 2))
    return np.divide(N1, sigma_tot, out=np.ones_like(N1), where=sigma_tot > 1e-30) - 1.0


def scan_observables(results, e_homo: float) -> dict:
    """Cross sections, delays and q for every polarisation of a scan.

    results: EnergyResult list of one channel set (same l_cont), in any order;
    they are sorted by energy.  Returns arrays over the sorted energies."""
    res = sorted(results, key=lambda r: r.E)
    E = np.array([r.E for r in res])
    k = np.sqrt(2.0 * E)
    omega = E - e_homo
    out = {"E": E, "k": k, "omega": omega}
    for s, (gauge, pol) in enumerate(SLOTS):
        D = np.stack([r.D[s] for r in res])
        out[f"sigma_{gauge}_{pol}"] = cross_section(k, D, omega, gauge)
        out[f"tau_{gauge}_{pol}"] = time_delay(k, D) if len(res) > 1 else np.zeros(1)
    for p, pol in enumerate("xyz"):
        DL = np.stack([r.D[p] for r in res])
        DV = np.stack([r.D[3 + p] for r in res])
        out[f"q_{pol}"] = q_sigma(DL, DV, omega)
        out[f"dphi_rms_{pol}"] = dphi_rms(DL, DV)
    for g, gauge in enumerate(("length", "velocity")):
        out[f"beta_{gauge}"] = beta(*(np.stack([r.D[3 * g + p] for r in res]) for p in range(3)))
    return out

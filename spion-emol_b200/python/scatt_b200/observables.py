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
(V,x) (V,y) (V,z).
"""
from __future__ import annotations

import numpy as np

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
    return out

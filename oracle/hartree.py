"""Hartree potential from density multipoles by the radial Poisson
integrals.  TEST INFRASTRUCTURE ONLY (the oracle for a device version of
this preprocessing step).

Restates preprocessing/src/potential/Hartree.hpp:71-246 (build_V_H) and the
cumulative integrator of preprocessing/src/sce/RadialGrid.hpp:63-100:

    V_lm(r) = 4 pi / (2l + 1) [ r^-(l+1) int_0^r rho_lm r'^(l+2) dr'
                              + r^l      int_r^R rho_lm r'^(1-l) dr' ]

on the uniform grid r_k = r0 + k dr, with the reference's guards: channels
above the overflow-safe l, and channels whose |rho_lm| stays below 1e-12,
are left at 0; a non-finite value is set to 0; at r = 0 the first term is
0, the second is 0 for l >= 1, and V_00(0) = 4 pi int_0^R rho_00 r' dr'.
The integrator is third order globally (each one-sided interval leaves h^4
times the third derivative / 24), although RadialGrid.hpp:69-70 calls it
fourth order.
"""
from __future__ import annotations

import math

import numpy as np


def cumulative_integrate(f: np.ndarray, dr: float) -> np.ndarray:
    """RadialGrid.hpp:84-100: I[0] = 0, I[k+1] = I[k] + h/12 (5 f_k + 8 f_k+1 - f_k+2),
    the last interval by the backward stencil h/12 (-f_N-3 + 8 f_N-2 + 5 f_N-1)."""
    n = f.shape[-1]
    if n < 3:
        raise RuntimeError("cumulative_integrate: need N >= 3")
    inc = np.empty(f.shape[:-1] + (n - 1,))
    inc[..., : n - 2] = (dr / 12.0) * (5.0 * f[..., : n - 2] + 8.0 * f[..., 1: n - 1] - f[..., 2:])
    inc[..., n - 2] = (dr / 12.0) * (-f[..., n - 3] + 8.0 * f[..., n - 2] + 5.0 * f[..., n - 1])
    out = np.zeros(f.shape)
    out[..., 1:] = np.cumsum(inc, axis=-1)
    return out


def l_safe(r: np.ndarray, l_max: int) -> int:
    """Hartree.hpp:98-139: the largest l for which r^l and r^(1-l) stay finite."""
    cap = l_max
    if r[-1] > 1.0:
        cap = min(cap, int(690.0 / math.log(r[-1])))
    pos = r[r > 0.0]
    if pos.size and pos[0] < 1.0:
        cap = min(cap, 1 + int(690.0 / math.log(1.0 / pos[0])))
    return cap


def build_V_H(rho_lm: np.ndarray, dr: float, l_max: int, r0: float = 0.0) -> np.ndarray:
    """Hartree.hpp:71-246: V_H (Nlm, Nr) from rho_lm (>= (l_max+1)^2 rows, Nr columns)."""
    n_lm = (l_max + 1) ** 2
    if rho_lm.shape[0] < n_lm:
        raise RuntimeError("build_V_H: rho_lm rows < (Lmax+1)^2")
    Nr = rho_lm.shape[1]
    r = r0 + np.arange(Nr) * dr
    V = np.zeros((n_lm, Nr))
    cap = l_safe(r, l_max)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for ch in range(n_lm):
            l = int(math.isqrt(ch))
            if l > cap:
                continue
            rho = rho_lm[ch]
            if np.max(np.abs(rho)) < 1e-12:
                continue
            pref = 4.0 * math.pi / (2.0 * l + 1.0)
            f_in = rho * r ** (l + 2)
            if l == 0:
                f_out = rho * r
            else:
                f_out = np.where(r <= 0.0, 0.0, rho * np.where(r <= 0.0, 1.0, r) ** (1 - l))
            I_in = cumulative_integrate(f_in, dr)
            I_out = cumulative_integrate(f_out, dr)
            term1 = np.where(r <= 0.0, 0.0, I_in / np.where(r <= 0.0, 1.0, r) ** (l + 1))
            v = pref * (term1 + r ** l * (I_out[-1] - I_out))
            v[~np.isfinite(v)] = 0.0
            if l == 0:
                v[0] = pref * I_out[-1]
            V[ch] = v
    return V

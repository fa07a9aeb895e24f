"""Potential cube V(r) of the oracle.

Restates src/scatt/Potentials.cpp:
  * compute_V_sigma_total ........ Potentials.cpp:40-88  (V_H + nuclear multipoles)
  * compute_U_polarization_at_r .. Potentials.cpp:111-129 (damped -a/2 r^-4, r_c = 1.5)
  * assemble_V_at ................ Potentials.cpp:324-365 (Gaunt contraction, V_pol,
                                   l(l+1)/(2 r^2)), r = r_min + ir*dr with r_min = 0
and src/angular/GauntSparse.hpp:130-222 for the Gaunt contraction
V_{mu',mu}(r) = sum_sigma V_sigma(r) G^R(mu', sigma, mu), |G| > 1e-15.

A second polarisation form, V_pol = -alpha / (2 (r^2 + r_c^2)^2), is
selectable (pol_form = 1); it is the adjoint benchmark's parametrisation and
is not in the reference.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

from . import angular


def v_sigma_total(inp, r: float, ir: int) -> np.ndarray:
    """Potentials.cpp:40-88 -- V_sigma(r) for sigma < n_exp = (2 l_cont + 1)^2."""
    l_exp = 2 * inp.l_cont
    n_exp = (l_exp + 1) ** 2
    V = np.zeros(n_exp)
    nH = min(n_exp, inp.V_H.shape[0])
    V[:nH] += inp.V_H[:nH, ir]
    for Z, x, y, z in inp.atoms:
        R = math.sqrt(x * x + y * y + z * z)
        th = ph = 0.0
        if R > 1e-14:
            th = math.acos(min(1.0, max(-1.0, z / R)))
            ph = math.atan2(y, x)
        rl, rg = min(r, R), max(r, R)
        for l in range(l_exp + 1):
            radial = (4.0 * math.pi / (2.0 * l + 1.0)) * rl**l / rg ** (l + 1)
            for m in range(-l, l + 1):
                if R < 1e-14:
                    Y = (1.0 / (2.0 * math.sqrt(math.pi))) if l == 0 else 0.0
                else:
                    Y = angular.real_Ylm(l, m, th, ph)
                if abs(Y) > 1e-15:
                    V[angular.lm_to_idx(l, m)] += -Z * radial * Y
    return V


def v_sigma_table(inp) -> np.ndarray:
    """V_sigma(r_ir) for every grid point, shape (n_exp, Nr); r = ir * dr.

    Same terms and accumulation order as v_sigma_total, vectorised over r.
    """
    l_exp = 2 * inp.l_cont
    n_exp = (l_exp + 1) ** 2
    r = np.arange(inp.Nr, dtype=np.float64) * inp.dr
    T = np.zeros((n_exp, inp.Nr))
    nH = min(n_exp, inp.V_H.shape[0])
    T[:nH] += inp.V_H[:nH, :]
    for Z, x, y, z in inp.atoms:
        R = math.sqrt(x * x + y * y + z * z)
        th = ph = 0.0
        if R > 1e-14:
            th = math.acos(min(1.0, max(-1.0, z / R)))
            ph = math.atan2(y, x)
        rl, rg = np.minimum(r, R), np.maximum(r, R)
        for l in range(l_exp + 1):
            with np.errstate(divide="ignore", invalid="ignore"):
                radial = (4.0 * math.pi / (2.0 * l + 1.0)) * np.power(rl, l) / np.power(rg, l + 1)
            for m in range(-l, l + 1):
                if R < 1e-14:
                    Y = (1.0 / (2.0 * math.sqrt(math.pi))) if l == 0 else 0.0
                else:
                    Y = angular.real_Ylm(l, m, th, ph)
                if abs(Y) > 1e-15:
                    T[angular.lm_to_idx(l, m)] += -Z * radial * Y
    T[:, r <= 1e-14] = 0.0
    return T


def gaunt_pairs(l_cont: int):
    """GauntSparse.hpp:130-180 -- sparse G(pair(mu', mu), sigma), mu >= mu'."""
    ch = (l_cont + 1) ** 2
    l_exp = 2 * l_cont
    n_exp = (l_exp + 1) ** 2
    rows, cols, vals = [], [], []
    for mu_p in range(ch):
        l2, m2 = angular.idx_to_lm(mu_p)
        for mu in range(mu_p, ch):
            l1, m1 = angular.idx_to_lm(mu)
            for ls in range(abs(l1 - l2), min(l1 + l2, l_exp) + 1):
                if (l1 + ls + l2) & 1:
                    continue
                for ms in angular.m3_candidates(m1, m2, ls):
                    G = angular.gaunt_real(l2, m2, ls, ms, l1, m1)
                    if abs(G) > 1e-15:
                        rows.append((mu_p, mu))
                        cols.append(angular.lm_to_idx(ls, ms))
                        vals.append(G)
    pairs = sorted(set(rows))
    pidx = {p: i for i, p in enumerate(pairs)}
    Gs = sp.csr_matrix((vals, ([pidx[p] for p in rows], cols)), shape=(len(pairs), n_exp))
    Gs.sort_indices()
    return np.array(pairs, dtype=np.int64).reshape(-1, 2), Gs


def v_pol(inp, r: float) -> float:
    """Potentials.cpp:111-129 (pol_form 0) or the adjoint benchmark form (pol_form 1)."""
    if inp.alpha_pol == 0.0 or r < 1.0e-6:
        return 0.0
    if inp.pol_form == 0:
        u = r / inp.r_c
        u6 = u**6
        damp = 1.0 - math.exp(-u6)
        return -0.5 * inp.alpha_pol * damp * damp / (r**4)
    return -inp.alpha_pol / (2.0 * (r * r + inp.r_c * inp.r_c) ** 2)


class VCube:
    """V(ir), N_ch x N_ch, assembled on demand (Potentials::V_at, ON_DEMAND mode)."""

    def __init__(self, inp):
        self.inp = inp
        self.ch = (inp.l_cont + 1) ** 2
        self.pairs, self.Gs = gaunt_pairs(inp.l_cont)
        self.vsig = v_sigma_table(inp)
        self.cent = np.array([angular.idx_to_lm(m)[0] for m in range(self.ch)], dtype=np.float64)
        self._cache = {}

    def get(self, ir: int) -> np.ndarray:
        if ir in self._cache:
            return self._cache[ir]
        inp = self.inp
        r = ir * inp.dr
        V = np.zeros((self.ch, self.ch))
        if r > 1e-14:
            flat = self.Gs @ self.vsig[:, ir]
            V[self.pairs[:, 0], self.pairs[:, 1]] = flat
            V[self.pairs[:, 1], self.pairs[:, 0]] = flat
            V[np.diag_indices(self.ch)] += v_pol(inp, r)
            inv_r2 = 1.0 / (r * r)
            V[np.diag_indices(self.ch)] += self.cent * (self.cent + 1.0) * 0.5 * inv_r2
        if len(self._cache) < 64:
            self._cache[ir] = V
        return V

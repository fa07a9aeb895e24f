"""Gradient checker for the adjoint.  TEST INFRASTRUCTURE ONLY.

The reference has no adjoint: the gradients asked for are the derivatives
of its forward path (sigma and tau per energy with respect to the two
parameters of the polarisation potential and to V_ll'(r) on the grid),
checked against central finite differences of that path.  Finite
differences can check the two scalars, but not a gradient over every grid
point and channel pair.  This module gives the exact derivative of the
oracle's forward path (solver.solve_energy): the same stages restated in
float64 torch on the CPU and differentiated by torch.autograd.  The tests
hold it to central differences of the numpy oracle, for (alpha, r_c) and
along random directions of V_ll'(r); it is then the checker for a device
adjoint.  Only the test suite imports it.

Parameters
  alpha, r_c  V_pol = -alpha / (2 (r^2 + r_c^2)^2) (pol_form 1), or the
              reference's damped form -alpha/2 (1 - exp(-(r/r_c)^6))^2 / r^4
              (pol_form 0, Potentials.cpp:111-129); added to the diagonal of
              V(n) at r = n dr for r >= 1e-6, like oracle.potentials.v_pol.
  dV          optional (Nr, N_mu, N_mu) tensor added to V(n).
Objectives
  sigma_L, sigma_V per polarisation and tau per energy, as
  oracle/observables.py states them (cross_section_delay.py:195-263).
Discrete choices -- a stability shift taken or not (SchurInverter.cpp:53-59),
closed channels (AsymptoticAmplitudes.cpp:173-212), the zero-coupling test of
KMatrixExtractor.cpp -- are made on detached values exactly as the oracle
makes them; the gradient is that of the branch taken.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import solver as O
from .bessel import riccati_j, riccati_y
from .observables import C_AU

F64 = torch.float64


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), dtype=F64)


def _sym(M):
    return 0.5 * (M + M.T)


def v_pol(r: float, alpha, r_c, pol_form: int):
    """oracle.potentials.v_pol with tensor parameters."""
    if r < 1.0e-6:
        return alpha * 0.0
    if pol_form == 0:
        u6 = (r / r_c) ** 6
        damp = 1.0 - torch.exp(-u6)
        return -0.5 * alpha * damp * damp / r ** 4
    return -alpha / (2.0 * (r * r + r_c * r_c) ** 2)


class Problem:
    """One setup (built without V_pol) and its energy-independent tensors."""

    def __init__(self, st: O.Setup, pol_form: int = 1):
        if st.inp.alpha_pol != 0.0:
            raise ValueError("build the setup with alpha_pol = 0; V_pol enters as a parameter")
        self.st = st
        self.pol_form = pol_form
        self.V0 = [_t(O.V_at(st, n)) for n in range(st.Nr)]
        self.Dinv = [_t(O.dinv_at(st, n)) for n in range(st.Nr)]
        self.B = [_t(O.B_at(st, n)) for n in range(st.Nr)]

    # V(n) with the parameters
    def V(self, n, alpha, r_c, dV):
        st = self.st
        r = n * st.dr
        V = self.V0[n]
        if r > 1e-14:
            V = V + v_pol(r, alpha, r_c, self.pol_form) * torch.eye(st.n_mu, dtype=F64)
        if dV is not None:
            V = V + dV[n]
        return V


def _shift(M):
    """SchurInverter.cpp:53-59: the decision on the detached values, the
    shift delta = W_min - lambda_min + margin as a function of M."""
    me = O.min_eig_fast(M.detach().numpy(), O.W_MIN)
    if me >= O.W_MIN:
        return M
    lam = torch.linalg.eigvalsh(M)[0]
    return M + (O.W_MIN - lam + O.SHIFT_MARGIN) * torch.eye(M.shape[0], dtype=F64)


def _sinv(P: Problem, E: float, n: int, V):
    """solver.sinv_at."""
    st = P.st
    h2_6 = st.dr * st.dr / 6.0
    A = (1.0 + h2_6 * E) * torch.eye(st.n_mu, dtype=F64) - h2_6 * V
    if n < O.STAB_N_MAX:
        A = _shift(_sym(A))
    if n < st.n_tr:
        B = P.B[n]
        S = A - (B * P.Dinv[n][None, :]) @ B.T
        if n < O.STAB_N_MAX:
            S = _shift(S)
    else:
        S = A
    return _sym(torch.linalg.inv(S))


def _winv_apply(P: Problem, n: int, Sinv, Z):
    """solver.winv_apply."""
    st = P.st
    Dinv = P.Dinv[n]
    Zp, Zf = Z[: st.n_mu], Z[st.n_mu:]
    tmp_f = Dinv[:, None] * Zf
    if n < st.n_tr:
        B = P.B[n]
        Yp = Sinv @ (Zp - B @ tmp_f)
        Yf = tmp_f - Dinv[:, None] * (B.T @ Yp)
    else:
        Yp = Sinv @ Zp
        Yf = tmp_f
    return torch.cat([Yp, Yf], dim=0)


def _analytic_init(P: Problem, E: float, n: int, Vn, Vn1):
    """solver.analytic_init: the psi block depends on diag V(n), diag V(n+1)."""
    st = P.st
    R0 = _t(O.analytic_init(st, E, n))          # the f block and the layout
    if n <= 0:
        return R0
    h = st.dr
    h2_6 = h * h / 6.0
    k = math.sqrt(2.0 * E)
    rn, rn1 = st.dr + n * h, st.dr + (n + 1) * h
    yn = _t(riccati_j(st.l_mu, k * rn))
    yn1 = _t(riccati_j(st.l_mu, k * rn1))
    Mn = 1.0 + h2_6 * (E - torch.diagonal(Vn))
    Mn1 = 1.0 + h2_6 * (E - torch.diagonal(Vn1))
    den = Mn1 * yn1
    ok = torch.abs(den.detach()) > 1e-300
    diag = torch.where(ok, (Mn * yn) / torch.where(ok, den, torch.ones_like(den)), torch.zeros_like(den))
    idx = torch.arange(st.n_mu)
    R = R0.clone()
    R[idx, idx] = diag
    return R


def _kme(P: Problem, E: float, Rinv_nM, n_match: int):
    """solver.kme_extract (K only)."""
    st = P.st
    Np, Nf = st.n_mu, st.Nf
    h = st.dr
    h2_12 = h * h / 12.0
    k = math.sqrt(2.0 * E)
    r_in, r_out = st.dr + n_match * h, st.dr + (n_match + 1) * h
    R = torch.linalg.inv(Rinv_nM)
    Rpp, Rpf, Rfp, Rff = R[:Np, :Np], R[:Np, Np:], R[Np:, :Np], R[Np:, Np:]
    if Nf == 0:
        S = R
    elif (np.linalg.norm(Rpf.detach().numpy()) < 1e-14 and np.linalg.norm(Rfp.detach().numpy()) < 1e-14):
        S = Rpp
    else:
        S = Rpp - Rpf @ torch.linalg.inv(Rff) @ Rfp
    S = _sym(S)
    l = st.l_mu
    lf = l.astype(np.float64)
    Jin, Jout = _t(riccati_j(l, k * r_in)), _t(riccati_j(l, k * r_out))
    Yin, Yout = _t(riccati_y(l, k * r_in)), _t(riccati_y(l, k * r_out))
    Win = _t(1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_in * r_in)))
    Wout = _t(1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_out * r_out)))
    A_mat = torch.diag(Wout * Jout) - S * (Win * Jin)[None, :]
    B_mat = S * (Win * Yin)[None, :] - torch.diag(Wout * Yout)
    return _sym(torch.linalg.solve(B_mat, A_mat))


def _aa(P: Problem, E: float, psi: dict):
    """solver.aa_extract (A and B)."""
    st = P.st
    Np = st.n_mu
    k = math.sqrt(2.0 * E)
    ns, ne = O.aa_window(st)
    r = st.dr + np.arange(ns, ne + 1) * st.dr
    Jc = np.array([riccati_j(int(l), k * r) for l in st.l_mu])
    Yc = np.array([riccati_y(int(l), k * r) for l in st.l_mu])
    c00, c01, c10, c11 = (np.zeros(Np) for _ in range(4))
    closed = np.zeros(Np, dtype=bool)
    for mu in range(Np):
        j, y = Jc[mu], Yc[mu]
        M = np.array([[j @ j, j @ y], [j @ y, y @ y]])
        det = M[0, 0] * M[1, 1] - M[0, 1] * M[1, 0]
        mx = np.max(np.abs(M))
        if not (abs(det) > 1e-20 * mx * mx):
            closed[mu] = True
            continue
        Mi = np.linalg.inv(M)
        c00[mu], c01[mu], c10[mu], c11[mu] = Mi[0, 0], Mi[0, 1], Mi[1, 0], Mi[1, 1]
    Pw = torch.stack([psi[n] for n in range(ns, ne + 1)])          # (nfit, Np, Np)
    YJ = torch.einsum("mi,imb->mb", _t(Jc), Pw)
    YY = torch.einsum("mi,imb->mb", _t(Yc), Pw)
    A = _t(c00)[:, None] * YJ + _t(c01)[:, None] * YY
    B = _t(c10)[:, None] * YJ + _t(c11)[:, None] * YY
    cl = torch.as_tensor(closed)[:, None]
    A = torch.where(cl, torch.eye(Np, dtype=F64), A)
    B = torch.where(cl, torch.zeros_like(B), B)
    return A, B


def _dme(P: Problem, A, B, psi: dict, n_lo: int, n_hi: int):
    """solver.dme_compute_six (D of the six slots)."""
    st = P.st
    n_pts = n_hi - n_lo
    Xi = O.xi_tables(st, n_lo, n_hi)
    rows = np.arange(n_lo, n_hi)
    r = st.dr + rows * st.dr
    w = _t(O.simpson(np.eye(n_pts), st.dr))                          # Simpson weights
    Psi = torch.stack([psi[int(ir)] for ir in rows])                  # (n_pts, Np, Np)
    M = torch.linalg.inv(A.to(torch.complex128) - 1j * B.to(torch.complex128)).conj().T
    mu_hi = min(st.n_mu, st.n_lambda)
    phi = _t(st.phi[:, rows, :mu_hi])                                 # (n_occ, n_pts, mu_hi)
    b_overlap = torch.einsum("r,arm,rmb->ba", w, phi, Psi[:, :mu_hi, :])   # (Np, n_occ)
    o = M @ b_overlap.to(torch.complex128)
    out = []
    for s, (g, q) in enumerate(O.SLOTS):
        rfac = r if g == "L" else np.ones_like(r)
        d_raw = torch.einsum("r,rm,rmb->b", w * _t(rfac), _t(Xi[s]), Psi)
        dcorr = np.array([O.simpson(rfac * np.sum(st.phi[a, rows, :mu_hi] * Xi[s][:, :mu_hi], axis=1), st.dr)
                          for a in range(st.n_occ)])
        D = M @ d_raw.to(torch.complex128) - o @ _t(st.spin * dcorr).to(torch.complex128)
        out.append(D)
    return out


def _forward(P: Problem, E: float, alpha, r_c, dV, n_last: int):
    """V(n), Sinv(n) for every n and Rinv(n) up to n_last (solver.solve_energy)."""
    st = P.st
    Nr, Nt = st.Nr, st.Nt
    Vs = [P.V(n, alpha, r_c, dV) for n in range(Nr)]
    Sinv = [_sinv(P, E, n, Vs[n]) for n in range(Nr)]
    ns = O.n_start(st)
    I = torch.eye(Nt, dtype=F64)
    Rinv = [None] * Nr
    for n in range(ns):
        Rinv[n] = _analytic_init(P, E, n, Vs[n], Vs[n + 1])
    prev = Rinv[ns - 1]
    for n in range(ns, n_last + 1):
        U = 12.0 * _winv_apply(P, n, Sinv[n], I) - 10.0 * I
        prev = _sym(torch.linalg.inv(U - prev))
        Rinv[n] = prev
    return Vs, Sinv, Rinv


def k_matrix(P: Problem, E: float, alpha, r_c, dV=None):
    """K of one energy (KMatrixExtractor at n_match = Nr - 2)."""
    n_match = P.st.Nr - 2
    _, _, Rinv = _forward(P, E, alpha, r_c, dV, n_match)
    return _kme(P, E, Rinv[n_match], n_match)


def dipoles(P: Problem, E: float, alpha, r_c, dV=None):
    """The six orthogonalised reduced dipoles D of one energy (solver.solve_energy)."""
    st = P.st
    Nr, Np, Nt = st.Nr, st.n_mu, st.Nt
    Vs, Sinv, Rinv = _forward(P, E, alpha, r_c, dV, Nr - 1)
    n_match = Nr - 2
    K = _kme(P, E, Rinv[n_match], n_match)
    k = math.sqrt(2.0 * E)
    rN = st.dr + (Nr - 1) * st.dr
    bc = torch.diag(_t(riccati_j(st.l_mu, k * rN))) + _t(riccati_y(st.l_mu, k * rN))[:, None] * K
    N = Nr - 1
    n_keep_hi = min(Nr - 1, max(1, st.n_tr - 1))
    asym_lo = N - O.N_ASYM + 1
    h2_6 = st.dr * st.dr / 6.0
    B_N = P.B[N]
    f_N = -(P.Dinv[N][:, None] * (B_N.T @ bc))
    Zp = bc + h2_6 * E * bc - h2_6 * Vs[N] @ bc + B_N @ f_N
    Z = torch.cat([Zp, torch.zeros(Nt - Np, Np, dtype=F64)], dim=0)
    psi = {N: bc}
    for n in range(N - 1, -1, -1):
        Z = Rinv[n] @ Z
        if n <= n_keep_hi or n >= asym_lo:
            psi[n] = _winv_apply(P, n, Sinv[n], Z)[:Np]
    A, B = _aa(P, E, psi)
    n_hi = min(Nr, n_keep_hi + 1)
    return _dme(P, A, B, psi, 0, n_hi)


def d_dk(k, f):
    """oracle.observables.d_dk over the first axis of a tensor."""
    n = len(k)
    out = [None] * n
    out[0] = (f[1] - f[0]) / (k[1] - k[0])
    out[n - 1] = (f[n - 1] - f[n - 2]) / (k[n - 1] - k[n - 2])
    for i in range(1, n - 1):
        hm, hp = k[i] - k[i - 1], k[i + 1] - k[i]
        out[i] = (hm * hm * f[i + 1] - hp * hp * f[i - 1] + (hp * hp - hm * hm) * f[i]) / (hm * hp * (hm + hp))
    return torch.stack(out)


def observables(P: Problem, Es, e_homo: float, alpha, r_c, dV=None):
    """sigma_{L,V} and tau per polarisation over the energies Es (ascending):
    a dict of (n_energy,) tensors keyed like scatt_b200.observables."""
    Es = [float(E) for E in Es]
    k = [math.sqrt(2.0 * E) for E in Es]
    Ds = [dipoles(P, E, alpha, r_c, dV) for E in Es]
    out = {}
    for s, (g, q) in enumerate(O.SLOTS):
        gauge = "length" if g == "L" else "velocity"
        pol = "xyz"[s % 3]
        D = torch.stack([Ds[e][s] for e in range(len(Es))])           # (n_energy, Np)
        s2 = torch.sum(torch.abs(D) ** 2, dim=1)
        om = torch.tensor([E - e_homo for E in Es], dtype=F64)
        kk = torch.tensor(k, dtype=F64)
        if gauge == "length":
            out[f"sigma_{gauge}_{pol}"] = 8.0 * math.pi * om / (C_AU * kk) * s2
        else:
            out[f"sigma_{gauge}_{pol}"] = 8.0 * math.pi / (C_AU * kk * om) * s2
        if len(Es) > 1:
            dD = d_dk(k, D) / kk[:, None]
            out[f"tau_{gauge}_{pol}"] = torch.sum(torch.conj(D) * dD, dim=1).imag / s2
    return out

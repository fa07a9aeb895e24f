"""Hand-written reverse pass of the Schur + Numerov recurrence, with R-ratio
checkpoints.  TEST INFRASTRUCTURE ONLY.

The reference has no adjoint.  This module states, in numpy, the reverse
pass a device adjoint performs for K (the output of the forward recurrence),
so that the device kernels can be checked stage by stage against it:

forward  (solver.sinv_at, solver.frp_step, solver.analytic_init)
  A(n)    = (1 + h^2 E / 6) I - h^2/6 V(n);  for n < 60: A <- shift(sym(A))
  S(n)    = A - B D^-1 B^T (n < n_tr; else A);  for n < 60: S <- shift(S)
  Sinv(n) = sym(S^-1)
  W^-1(n) = [[Sinv, Sinv P], [P^T Sinv, D^-1 + P^T Sinv P]],  P = -B D^-1
  Rinv(n) = sym((12 W^-1(n) - 10 I - Rinv(n-1))^-1),  n >= n_start
  Rinv(n_start - 1) from the analytic start (diagonal in the psi block)
  shift(M) = M + (W_min - lambda_min(M) + margin) I when lambda_min < W_min
reverse, for Rbar = dJ/dRinv(n):
  Xbar = sym(Rbar);  Rbar_n = -X^T Xbar X^T  with X = (12 W^-1 - 10 I - Rinv(n-1))^-1
  dJ/dRinv(n-1) += -Rbar_n;  Wbar = 12 Rbar_n
  Sinvbar = Wbar_pp + Wbar_pf P^T + P Wbar_fp + P Wbar_ff P^T
  Sbar = -Y^T sym(Sinvbar) Y^T  with Y = S^-1
  through a shift:  Mbar <- Mbar - tr(Mbar) v v^T  (v: eigenvector of lambda_min)
  Vbar(n) = -h^2/6 sym(Abar)  (sym only where the forward symmetrised A)
  analytic start: d R_mumu / d V(n)_mumu = -h^2/6 y_n / (M_n+1 y_n+1),
                  d R_mumu / d V(n+1)_mumu = h^2/6 M_n y_n / (M_n+1^2 y_n+1)

Memory: the forward pass keeps Rinv only every `segment` steps (256 by
default); the reverse pass recomputes each segment's Rinv(n), Sinv(n) and
inverses from its checkpoint, then walks it backward.  The result does not
depend on the segment length (the recomputation repeats the same
arithmetic), which the tests check, together with agreement with the
autograd gradient of oracle/adjoint.py.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla

from . import solver as O
from .bessel import riccati_j

SEGMENT = 256


def _sym(M):
    return 0.5 * (M + M.T)


def _shift_tape(M):
    """solver.stability_shift, also returning the eigenvector of lambda_min
    when the shift is taken (None otherwise)."""
    me = O.min_eig_fast(M, O.W_MIN)
    if me >= O.W_MIN:
        return M, None
    w, V = sla.eigh(M, lower=True)
    M = M.copy()
    M[np.diag_indices_from(M)] += O.W_MIN - w[0] + O.SHIFT_MARGIN
    return M, V[:, 0]


def _shift_reverse(Mbar, v):
    if v is None:
        return Mbar
    return Mbar - np.trace(Mbar) * np.outer(v, v)


class Step:
    """Sinv(n) with what its reverse needs."""

    def __init__(self, st, E, n, V):
        h2_6 = st.dr * st.dr / 6.0
        A = np.eye(st.n_mu) * (1.0 + h2_6 * E) - h2_6 * V
        self.vA = self.vS = None
        if n < O.STAB_N_MAX:
            A, self.vA = _shift_tape(_sym(A))
        if n < st.n_tr:
            B = O.B_at(st, n)
            S = A - (B * O.dinv_at(st, n)[None, :]) @ B.T
            if n < O.STAB_N_MAX:
                S, self.vS = _shift_tape(S)
        else:
            S = A
        self.n = n
        self.Y = np.linalg.inv(S)
        self.Sinv = _sym(self.Y)

    def Vbar(self, st, Sinv_bar):
        """dJ/dV(n) from dJ/dSinv(n)."""
        Sbar = -self.Y.T @ _sym(Sinv_bar) @ self.Y.T
        if self.n < st.n_tr:
            Abar = _shift_reverse(Sbar, self.vS) if self.n < O.STAB_N_MAX else Sbar
        else:
            Abar = Sbar
        if self.n < O.STAB_N_MAX:
            Abar = _sym(_shift_reverse(Abar, self.vA))
        return -(st.dr * st.dr / 6.0) * Abar


def _winv(st, n, Sinv):
    return O.winv_apply(st, n, Sinv, np.eye(st.Nt))


def _sinv_bar(st, n, Wbar):
    """dJ/dSinv(n) from dJ/dW^-1(n)."""
    Np = st.n_mu
    if n >= st.n_tr:
        return Wbar[:Np, :Np].copy()
    P = -(O.B_at(st, n) * O.dinv_at(st, n)[None, :])
    return Wbar[:Np, :Np] + Wbar[:Np, Np:] @ P.T + P @ Wbar[Np:, :Np] + P @ Wbar[Np:, Np:] @ P.T


def _analytic(st, E, n, V_of):
    """solver.analytic_init with the psi block recomputed from V_of."""
    R = O.analytic_init(st, E, n)
    h = st.dr
    h2_6 = h * h / 6.0
    k = math.sqrt(2.0 * E)
    rn, rn1 = st.dr + n * h, st.dr + (n + 1) * h
    yn, yn1 = riccati_j(st.l_mu, k * rn), riccati_j(st.l_mu, k * rn1)
    Mn = 1.0 + h2_6 * (E - np.diag(V_of(n)))
    Mn1 = 1.0 + h2_6 * (E - np.diag(V_of(n + 1)))
    den = Mn1 * yn1
    ok = np.abs(den) > 1e-300
    idx = np.arange(st.n_mu)
    R[idx, idx] = np.where(ok, Mn * yn / np.where(ok, den, 1.0), 0.0)
    return R, (yn, yn1, Mn, Mn1, ok)


class Recurrence:
    """Forward recurrence to n_last with checkpoints, and its reverse."""

    def __init__(self, st, E, V_of, n_last=None, segment=SEGMENT):
        self.st, self.E, self.V_of = st, E, V_of
        self.segment = max(1, int(segment))
        self.ns = O.n_start(st)
        self.n_last = st.Nr - 2 if n_last is None else n_last
        self.start, self.start_tape = _analytic(st, E, self.ns - 1, V_of)
        self.checkpoints = {self.ns - 1: self.start}
        prev = self.start
        for n in range(self.ns, self.n_last + 1):
            prev, _, _ = self._step(n, prev)
            if (n - (self.ns - 1)) % self.segment == 0:
                self.checkpoints[n] = prev
        self.Rinv_last = prev

    def _step(self, n, prev):
        stp = Step(self.st, self.E, n, self.V_of(n))
        I = np.eye(self.st.Nt)
        X = np.linalg.inv(12.0 * _winv(self.st, n, stp.Sinv) - 10.0 * I - prev)
        return _sym(X), X, stp

    def reverse(self, Rbar_last):
        """dJ/dV(n) for every n (an (Nr, N_mu, N_mu) array) from dJ/dRinv(n_last)."""
        st = self.st
        Vbar = np.zeros((st.Nr, st.n_mu, st.n_mu))
        Rbar = Rbar_last
        bounds = sorted(self.checkpoints)
        for c in reversed(bounds):
            hi = min(c + self.segment, self.n_last)
            if hi <= c:
                continue
            # recompute the segment (c, hi] from its checkpoint
            prev = self.checkpoints[c]
            tape = []
            for n in range(c + 1, hi + 1):
                Rn, X, stp = self._step(n, prev)
                tape.append((X, stp))
                prev = Rn
            for n in range(hi, c, -1):
                X, stp = tape[n - c - 1]
                Rbar_n = -X.T @ _sym(Rbar) @ X.T
                Vbar[n] += stp.Vbar(st, _sinv_bar(st, n, 12.0 * Rbar_n))
                Rbar = -Rbar_n                                # dJ/dRinv(n-1)
        # the analytic start Rinv(n_start - 1)
        n0 = self.ns - 1
        if n0 >= 1:
            yn, yn1, Mn, Mn1, ok = self.start_tape
            h2_6 = st.dr * st.dr / 6.0
            d = np.diag(Rbar)[: st.n_mu]
            g_n = np.where(ok, -h2_6 * yn / np.where(ok, Mn1 * yn1, 1.0), 0.0)
            g_n1 = np.where(ok, h2_6 * Mn * yn / np.where(ok, Mn1 * Mn1 * yn1, 1.0), 0.0)
            idx = np.arange(st.n_mu)
            Vbar[n0][idx, idx] += d * g_n
            Vbar[n0 + 1][idx, idx] += d * g_n1
        return Vbar

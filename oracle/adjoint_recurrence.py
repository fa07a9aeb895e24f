"""Hand-written reverse pass of the Schur + Numerov recurrence, with R-ratio
checkpoints.  TEST INFRASTRUCTURE ONLY.

The reference has no adjoint.  This module states, in numpy, the reverse
pass a device adjoint performs -- for K (Recurrence) and for the six
dipoles through the back sweep (DipoleAdjoint) -- so that the device
kernels can be checked stage by stage against it:

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
import torch

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
    if n <= 0:                                   # Rinv(0) = 0, independent of V
        return R, None
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


# ------------------------------------------------------------------ dipoles
def _rows(st, n_hi):
    """L(n), n < n_hi: (n_hi, N_mu, 6 + n_occ).  Column s < 6 holds the Simpson
    weight x (r or 1) x Xi_s(n, mu) of slot s; column 6 + a the weight x
    phi_a(n, mu) of occupied orbital a (solver.dme_compute_six), so that
    d_raw[s] = Q[s] and b_overlap[:, a] = Q[6 + a] for Q = sum_n L(n)^T psi_n."""
    Xi = O.xi_tables(st, 0, n_hi)
    rows = np.arange(n_hi)
    r = st.dr + rows * st.dr
    w = O.simpson(np.eye(n_hi), st.dr)
    mu_hi = min(st.n_mu, st.n_lambda)
    L = np.zeros((n_hi, st.n_mu, 6 + st.n_occ))
    for s, (g, q) in enumerate(O.SLOTS):
        L[:, :, s] = (w * (r if g == "L" else 1.0))[:, None] * Xi[s]
    for a in range(st.n_occ):
        L[:, :mu_hi, 6 + a] = w[:, None] * st.phi[a, rows, :mu_hi]
    return L


class DipoleAdjoint:
    """Forward solve of one energy up to the six dipoles, and its reverse.

    forward, n = 0 .. N-1 (N = Nr - 1), one state (Rinv(n), G(n)):
      Rinv(n) = analytic start (n < n_start) or the recurrence
      G(n)    = Rinv(n)^T (G(n-1) + W^-1(n)^T E_psi L(n)),  G(-1) = 0
    so that Q = sum_n L(n)^T psi_n = G(N-1)^T Z_N (+ L(N)^T psi_N when the
    dipole rows reach N): the back sweep of the dipole rows is never run.
    The fit window of the asymptotic amplitudes (at most 300 points below N)
    is swept explicitly from Z_N.  (Rinv, G) is kept every `segment` steps.

    reverse, from dJ/dD by autograd of the small stages (dipole algebra,
    the fit, K extraction), then one downward sweep over n that recomputes
    each segment from its checkpoint:
      Rbar(n) = chain + H(n) Gbar(n)^T [+ fit-window term] [+ K term at Nr-2]
      Hbar(n) = Rinv(n) Gbar(n);  Gbar(n-1) = Hbar(n)
      Wbar(n) = E_psi L(n) Hbar(n)^T + 12 Rbar_n [+ fit-window term]
    and Wbar(n) -> Sinvbar(n) -> Vbar(n) as in Recurrence.reverse.
    """

    def __init__(self, st, E, V_of, segment=SEGMENT):
        self.st, self.E, self.V_of = st, E, V_of
        self.segment = max(1, int(segment))
        self.ns = O.n_start(st)
        Nr, Np, Nt = st.Nr, st.n_mu, st.Nt
        self.N = N = Nr - 1
        self.n_match = Nr - 2                    # KMatrixExtractor's matching point
        self.n_keep_hi = min(Nr - 1, max(1, st.n_tr - 1))
        self.n_hi = min(Nr, self.n_keep_hi + 1)
        self.L = _rows(st, self.n_hi)
        self.Ls = self.L.shape[2]
        self.wlo, self.whi = O.aa_window(st)
        # forward sweep
        self.checkpoints = {-1: (None, np.zeros((Nt, self.Ls)))}
        self.window = {}
        prev, G = None, np.zeros((Nt, self.Ls))
        for n in range(N):
            Rn, X, stp, Winv, H, G = self._step(n, prev, G)
            if n == self.n_match:
                self.Rinv_match = Rn
            if n >= self.wlo:
                self.window[n] = (Rn, stp, Winv)
            prev = Rn
            if (n + 1) % self.segment == 0:
                self.checkpoints[n] = (Rn, G)
        self.G_last = G
        # K, psi_N, Z_N
        h2_6 = st.dr * st.dr / 6.0
        self.K = O.kme_extract(st, E, self.Rinv_match, self.n_match)["K"]
        self.bc = O.psi_boundary(st, E, self.K)
        B_N = O.B_at(st, N)
        self.Gamma = ((1.0 + h2_6 * E) * np.eye(Np) - h2_6 * V_of(N)
                      - (B_N * O.dinv_at(st, N)[None, :]) @ B_N.T)
        self.Z_N = np.zeros((Nt, Np))
        self.Z_N[:Np] = self.Gamma @ self.bc
        self.Q = self.G_last.T @ self.Z_N
        if self.n_hi == Nr:
            self.Q += self.L[N].T @ self.bc
        # the fit window, swept down from Z_N
        self.Zw = {N: self.Z_N}
        self.psi_w = {}
        for m in range(N - 1, self.wlo - 1, -1):
            Rm, stp, Winv = self.window[m]
            self.Zw[m] = Rm @ self.Zw[m + 1]
            if m <= self.whi:
                self.psi_w[m] = (Winv @ self.Zw[m])[:Np]
        self.A, self.B = self._aa_torch({m: torch.as_tensor(p) for m, p in self.psi_w.items()})
        self.A, self.B = self.A.numpy(), self.B.numpy()

    # ---- pieces
    def _step(self, n, prev, G):
        st = self.st
        stp = Step(st, self.E, n, self.V_of(n))
        Winv = _winv(st, n, stp.Sinv)
        if n < self.ns:
            Rn, _ = _analytic(st, self.E, n, self.V_of)
            X = None
        else:
            X = np.linalg.inv(12.0 * Winv - 10.0 * np.eye(st.Nt) - prev)
            Rn = _sym(X)
        H = G.copy()
        if n < self.n_hi:
            H += Winv.T[:, : st.n_mu] @ self.L[n]
        return Rn, X, stp, Winv, H, Rn.T @ H

    def _aa_torch(self, psi):
        from .adjoint import _aa
        return _aa(self._problem(), self.E, psi)

    def _problem(self):
        """The torch tables of the small stages (V_pol, if any, lives in V_of)."""
        from .adjoint import Problem
        if not hasattr(self, "_P"):
            self._P = Problem(self.st)
        return self._P

    def dipoles_torch(self, A, B, Q):
        """The dipole algebra of solver.dme_compute_six from (A, B, Q)."""
        st = self.st
        rows = np.arange(self.n_hi)
        r = st.dr + rows * st.dr
        Xi = O.xi_tables(st, 0, self.n_hi)
        mu_hi = min(st.n_mu, st.n_lambda)
        M = torch.linalg.inv(A.to(torch.complex128) - 1j * B.to(torch.complex128)).conj().T
        o = M @ Q[6:].T.to(torch.complex128)
        out = []
        for s, (g, q) in enumerate(O.SLOTS):
            rfac = r if g == "L" else np.ones_like(r)
            dcorr = np.array([O.simpson(rfac * np.sum(st.phi[a, rows, :mu_hi] * Xi[s][:, :mu_hi], axis=1), st.dr)
                              for a in range(st.n_occ)])
            out.append(M @ Q[s].to(torch.complex128)
                       - o @ torch.as_tensor(st.spin * dcorr, dtype=torch.complex128))
        return out

    def dipoles(self):
        t = lambda a: torch.as_tensor(a, dtype=torch.float64)
        return [d.numpy() for d in self.dipoles_torch(t(self.A), t(self.B), t(self.Q))]

    # ---- reverse
    def reverse(self, objective):
        """dJ/dV(n), an (Nr, N_mu, N_mu) array, for J = objective(list of the six D)."""
        from .adjoint import _kme
        st = self.st
        Np, Nt, N = st.n_mu, st.Nt, self.N
        h2_6 = st.dr * st.dr / 6.0
        Vbar = np.zeros((st.Nr, Np, Np))
        # small stages by autograd: dipole algebra and the fit
        tA = torch.tensor(self.A, requires_grad=True)
        tB = torch.tensor(self.B, requires_grad=True)
        tQ = torch.tensor(self.Q, requires_grad=True)
        Abar, Bbar, Qbar = torch.autograd.grad(objective(self.dipoles_torch(tA, tB, tQ)), (tA, tB, tQ))
        Qbar = Qbar.numpy()
        tpsi = {m: torch.tensor(p, requires_grad=True) for m, p in self.psi_w.items()}
        A2, B2 = self._aa_torch(tpsi)
        ms = sorted(tpsi)
        gpsi = torch.autograd.grad((A2, B2), [tpsi[m] for m in ms], grad_outputs=(Abar, Bbar), allow_unused=True)
        psibar = {m: (g.numpy() if g is not None else np.zeros((Np, Np))) for m, g in zip(ms, gpsi)}
        # the fit window, upward: Zbar(m+1) += Rinv(m)^T Zbar(m)
        Rbar_w, Wbar_w = {}, {}
        carry = np.zeros((Nt, Np))
        for m in range(self.wlo, N):
            Rm, stp, Winv = self.window[m]
            Zbar = carry.copy()
            if m in psibar:
                Zbar += Winv.T[:, :Np] @ psibar[m]
                Wb = np.zeros((Nt, Nt))
                Wb[:Np] = psibar[m] @ self.Zw[m].T
                Wbar_w[m] = Wb
            Rbar_w[m] = Zbar @ self.Zw[m + 1].T
            carry = Rm.T @ Zbar
        ZbarN = carry + self.G_last @ Qbar
        bcbar = np.zeros((Np, Np))
        if self.n_hi == st.Nr:
            bcbar += self.L[N] @ Qbar
        bcbar += self.Gamma.T @ ZbarN[:Np]
        Vbar[N] += -h2_6 * ZbarN[:Np] @ self.bc.T
        rN = st.dr + N * st.dr
        Kbar = riccati_y_vec(st.l_mu, math.sqrt(2.0 * self.E) * rN)[:, None] * bcbar
        leaf = torch.tensor(self.Rinv_match, requires_grad=True)
        Rbar_kme, = torch.autograd.grad(_kme(self._problem(), self.E, leaf, self.n_match), (leaf,),
                                        grad_outputs=(torch.as_tensor(Kbar),))
        Rbar_kme = Rbar_kme.numpy()
        # the downward sweep, segment by segment
        Gbar = self.Z_N @ Qbar.T
        Rbar_chain = np.zeros((Nt, Nt))
        for c in sorted(self.checkpoints, reverse=True):
            hi = min(c + self.segment, N - 1)
            if hi <= c:
                continue
            prev, G = self.checkpoints[c]
            tape = {}
            for n in range(c + 1, hi + 1):
                Rn, X, stp, Winv, H, G = self._step(n, prev, G)
                tape[n] = (Rn, X, stp, H)
                prev = Rn
            for n in range(hi, c, -1):
                Rn, X, stp, H = tape[n]
                Rbar = Rbar_chain + H @ Gbar.T
                if n in Rbar_w:
                    Rbar = Rbar + Rbar_w[n]
                if n == self.n_match:
                    Rbar = Rbar + Rbar_kme
                Hbar = Rn @ Gbar
                Wbar = np.zeros((Nt, Nt))
                if n < self.n_hi:
                    Wbar[:Np] += self.L[n] @ Hbar.T
                if n in Wbar_w:
                    Wbar += Wbar_w[n]
                Gbar = Hbar
                if X is not None:
                    Rbar_n = -X.T @ _sym(Rbar) @ X.T
                    Wbar += 12.0 * Rbar_n
                    Rbar_chain = -Rbar_n
                else:
                    Rbar_chain = np.zeros((Nt, Nt))
                    if n >= 1:
                        _, (yn, yn1, Mn, Mn1, ok) = _analytic(st, self.E, n, self.V_of)
                        d = np.diag(Rbar)[:Np]
                        idx = np.arange(Np)
                        Vbar[n][idx, idx] += d * np.where(ok, -h2_6 * yn / np.where(ok, Mn1 * yn1, 1.0), 0.0)
                        Vbar[n + 1][idx, idx] += d * np.where(
                            ok, h2_6 * Mn * yn / np.where(ok, Mn1 * Mn1 * yn1, 1.0), 0.0)
                Vbar[n] += stp.Vbar(st, _sinv_bar(st, n, Wbar))
        return Vbar


def riccati_y_vec(l, x):
    from .bessel import riccati_y
    return np.asarray(riccati_y(l, x), dtype=np.float64)

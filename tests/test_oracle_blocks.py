"""The oracle's building blocks against the acceptance checks of the
reference's component tests (thresholds as there):

  src/tests/test_w_inverse_operator.cpp (1) W^-1 from the Schur structure ==
      LU inverse of the assembled W (W built as build_W_unshifted, :74-111),
      (3) W (W^-1 Z) == Z, (4) W^-1 symmetric, (5) past n_transition W^-1 is
      block-diagonal [Sinv, diag(1/D_clamp)];
  src/tests/test_schur_inverter.cpp  Sinv S == I, Sinv symmetric;
  src/tests/test_exchange_coupling.cpp  the CSR exchange coupling == the
      triple loop sum_lambda G(mu, lambda, sigma) chi_{i,lambda}(r);
  src/tests/test_lapack_inverse.cpp  A A^-1 = I and agreement with a
      partial-pivot LU inverse (1e-11), in both LAPACK builds;
  src/tests/test_sinv_symmetric_inverse.cpp  the dsytrf/dsytri Sinv exactly
      symmetric, Sinv S = I and within 1e-10 of the symmetrised LU inverse;
  src/tests/test_forward_r_propagator.cpp, test_back_propagator.cpp  (below).
"""
import dataclasses
import math

import numpy as np
import pytest

from oracle import angular
from oracle import solver as O
from scatt_b200 import synth


@pytest.fixture(scope="module", params=["h2", "h2o"])
def setup(request):
    if request.param == "h2":
        inp = synth.h2_like(Nr=801, dr=0.05, l_cont=2)
    else:
        inp = synth.h2o_like(Nr=601, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)
    return O.make_setup(inp)


def assembled_W(st, E, n):
    """W(n) = [[I + h^2/6 (E - V(n)), B], [B^T, diag(D)]], D clamped at W_min."""
    h2_6 = st.dr * st.dr / 6.0
    Np = st.n_mu
    W = np.zeros((st.Nt, st.Nt))
    W[:Np, :Np] = (1.0 + h2_6 * E) * np.eye(Np) - h2_6 * O.V_at(st, n)
    W[Np:, Np:] = np.diag(1.0 / O.dinv_at(st, n))
    B = O.B_at(st, n)
    W[:Np, Np:] = B
    W[Np:, :Np] = B.T
    return W


def materialize(st, E, n):
    return O.winv_apply(st, n, O.sinv_at(st, E, n), np.eye(st.Nt))


def test_w_inverse_operator(setup):
    st = setup
    E = 0.7
    rng = np.random.default_rng(42)
    for n in (O.STAB_N_MAX, 200, st.n_tr - 5, st.Nr - 2):
        M = materialize(st, E, n)
        Wn = assembled_W(st, E, n)
        ref = np.linalg.inv(Wn)
        assert np.max(np.abs(M - ref)) < 1e-9                              # (1)
        Z = rng.standard_normal((st.Nt, 3))
        Y = O.winv_apply(st, n, O.sinv_at(st, E, n), Z)
        assert np.max(np.abs(Wn @ Y - Z)) / np.max(np.abs(Z)) < 1e-10      # (3)
        assert np.max(np.abs(M - M.T)) / np.max(np.abs(M)) < 1e-12         # (4)


def test_w_inverse_block_diagonal_past_transition(setup):
    st = dataclasses.replace(setup, n_tr=min(setup.n_tr, 300))
    n = st.n_tr + 50
    E = 0.7
    M = materialize(st, E, n)
    Np = st.n_mu
    assert np.max(np.abs(M[:Np, :Np] - O.sinv_at(st, E, n))) < 1e-12
    assert np.max(np.abs(M[Np:, Np:] - np.diag(O.dinv_at(st, n)))) < 1e-12
    assert max(np.max(np.abs(M[:Np, Np:])), np.max(np.abs(M[Np:, :Np]))) < 1e-12


def test_schur_inverse(setup):
    st = setup
    E = 1.1
    h2_6 = st.dr * st.dr / 6.0
    for n in (O.STAB_N_MAX, 150, st.n_tr - 5):
        A = (1.0 + h2_6 * E) * np.eye(st.n_mu) - h2_6 * O.V_at(st, n)
        B = O.B_at(st, n)
        S = A - (B * O.dinv_at(st, n)[None, :]) @ B.T
        Sinv = O.sinv_at(st, E, n)
        assert np.max(np.abs(Sinv @ S - np.eye(st.n_mu))) < 1e-10
        assert np.array_equal(Sinv, Sinv.T)


def test_exchange_coupling_equals_triple_loop(setup):
    st = setup
    G = angular.build_G_vector(st.n_mu, st.n_lambda, st.n_sigma)
    for ir in (5, 40, st.n_tr // 2, st.n_tr - 1):
        Q = O.exchange_Q(st, ir)
        r = ir * st.dr
        ref = np.zeros_like(Q)
        chi = st.chi_r[:, :, ir]                       # (n_occ, n_lambda)
        for mu, la, sg, g in G:
            for i in range(st.n_occ):
                ref[mu, i * st.n_sigma + sg] += g * chi[i, la]
        ref *= 2.0 * math.sqrt(2.0 * math.pi) / r
        scale = max(np.max(np.abs(ref)), 1e-300)
        assert np.max(np.abs(Q - ref)) / scale < 1e-12


def _riccati_j(l, x):
    from scipy.special import spherical_jn
    return x * spherical_jn(l, x)


def test_forward_analytic_start():
    """test_forward_r_propagator.cpp (1): Rinv(n) for 1 <= n < n_start is the
    diagonal (M_n y_n) / (M_{n+1} y_{n+1}), off-diagonal zero (1e-14);
    r_n = r_min + n h with r_min = h, V at index n, y = x j_l(x) for the
    continuum channels and r^(l+1) for the exchange channels (:121-166)."""
    inp = synth.h2_like(Nr=201, dr=0.05, l_cont=10)
    st = O.make_setup(inp)
    E = 0.5
    h = st.dr
    h2_6, h2_12 = h * h / 6.0, h * h / 12.0
    k = math.sqrt(2.0 * E)
    ns = O.n_start(st)
    assert ns > 3
    for n in range(1, ns):
        R = O.analytic_init(st, E, n)
        rn, rn1 = h + n * h, h + (n + 1) * h
        Vn, Vn1 = O.V_at(st, n), O.V_at(st, n + 1)
        ref = np.zeros(st.Nt)
        for mu in range(st.n_mu):
            l = int(st.l_mu[mu])
            Mn, Mn1 = 1.0 + h2_6 * (E - Vn[mu, mu]), 1.0 + h2_6 * (E - Vn1[mu, mu])
            den = Mn1 * _riccati_j(l, k * rn1)
            if abs(den) > 1e-300:
                ref[mu] = Mn * _riccati_j(l, k * rn) / den
        for f in range(st.Nf):
            l = int(st.l_sigma_f[f])
            Mn = max(1.0 - h2_12 * l * (l + 1) / (rn * rn), O.W_MIN)
            Mn1 = max(1.0 - h2_12 * l * (l + 1) / (rn1 * rn1), O.W_MIN)
            den = Mn1 * rn1 ** (l + 1)
            if abs(den) > 1e-300:
                ref[st.n_mu + f] = Mn * rn ** (l + 1) / den
        off = R - np.diag(np.diag(R))
        assert np.max(np.abs(off)) == 0.0
        assert np.max(np.abs(np.diag(R) - ref)) < 1e-14


def test_forward_recursion_gold_standard(setup):
    """test_forward_r_propagator.cpp (2)-(3): the recursion against an
    independent path (LU inverse of the assembled W, then of 12 W^-1 - 10 I -
    Rinv_prev, symmetrised; :170-205) to 1e-8, and symmetric to 1e-12."""
    st = setup
    E = 0.9
    ns = O.n_start(st)
    I = np.eye(st.Nt)
    prev_o = O.analytic_init(st, E, ns - 1)
    prev_r = prev_o.copy()
    probes = {ns, ns + 1, ns + 5, 50, 200, st.Nr - 2, st.Nr - 1}
    worst = 0.0
    for n in range(ns, st.Nr):
        prev_o = O.frp_step(st, n, O.sinv_at(st, E, n), prev_o)
        Wi = np.linalg.inv(assembled_W(st, E, n)) if n >= O.STAB_N_MAX else \
            O.winv_apply(st, n, O.sinv_at(st, E, n), I)
        Rn = np.linalg.inv(12.0 * Wi - 10.0 * I - prev_r)
        prev_r = 0.5 * (Rn + Rn.T)
        if n in probes:
            worst = max(worst, np.max(np.abs(prev_o - prev_r)) / np.max(np.abs(prev_r)))
            assert np.all(np.isfinite(prev_o))
            assert np.max(np.abs(prev_o - prev_o.T)) / np.max(np.abs(prev_o)) < 1e-12
    assert worst < 1e-8


def test_back_propagation_checks():
    """test_back_propagator.cpp (1) the three-point Numerov identity
    W_{n+1} Y_{n+1} - (12 I - 10 W_n) Y_n + W_{n-1} Y_{n-1} = 0 (1e-8 rel),
    (2) psi_N == psi_boundary (1e-14), (3) psi_0 = 0 (1e-12), (4) psi_n close
    to J_n + Y_n K near the outer edge (1e-1 rel)."""
    inp = synth.h2_like(Nr=801, dr=0.05, l_cont=2)
    st = O.make_setup(inp)
    E = 0.8
    r = O.solve_energy(st, E, keep_rinv=True, keep_psi=True)
    N, Np = st.Nr - 1, st.n_mu
    bc = O.psi_boundary(st, E, r.K_kme)
    assert np.max(np.abs(r.psi_keep[N] - bc)) < 1e-14
    assert np.max(np.abs(r.psi_keep[0])) < 1e-12
    k = math.sqrt(2.0 * E)
    from scipy.special import spherical_jn, spherical_yn
    worst = 0.0
    for n in (N - 1, N - 2, N - 5, N - 10, N - 50, N - 100):
        rn = st.dr + n * st.dr
        lv = st.l_mu.astype(int)
        J = np.diag(k * rn * spherical_jn(lv, k * rn))
        Y = np.diag(k * rn * spherical_yn(lv, k * rn))
        ans = J + Y @ r.K_kme
        worst = max(worst, np.max(np.abs(r.psi_keep[n] - ans)) / np.max(np.abs(ans)))
    assert worst < 1e-1
    # backward sweep with the full Y = W^-1 Z (psi and f) for the identity
    h2_6 = st.dr * st.dr / 6.0
    B_N = O.B_at(st, N)
    f_N = -(O.dinv_at(st, N)[:, None] * (B_N.T @ bc))
    Z = np.zeros((st.Nt, Np))
    Z[:Np] = bc + h2_6 * E * bc - h2_6 * O.V_at(st, N) @ bc + B_N @ f_N
    Ys = {}
    probe = 300
    for n in range(N - 1, probe - 2, -1):
        Z = r.rinv[n] @ Z
        if n <= probe + 1:
            Ys[n] = O.winv_apply(st, n, O.sinv_at(st, E, n), Z)
    I = np.eye(st.Nt)
    Wp, Wn, Wq = (assembled_W(st, E, m) for m in (probe - 1, probe, probe + 1))
    res = Wq @ Ys[probe + 1] - (12.0 * I - 10.0 * Wn) @ Ys[probe] + Wp @ Ys[probe - 1]
    scale = max(np.max(np.abs(Ys[m])) for m in (probe - 1, probe, probe + 1))
    assert np.max(np.abs(res)) / scale < 1e-8


@pytest.mark.parametrize("build", ["eigen", "mkl"])
def test_lapack_inverse(monkeypatch, build):
    """test_lapack_inverse.cpp: for n in {1, 4, 17, 49, 121, 256}, on
    X^T X + n I and X + n I with X uniform in [-1, 1],
    ||A A^-1 - I||_inf / max(||A||_inf, 1) < 1e-11, and the inverse within
    1e-11 (relative) of a partial-pivot LU inverse."""
    monkeypatch.setattr(O, "BUILD", build)
    rng = np.random.default_rng(0xBEEF)
    for n in (1, 4, 17, 49, 121, 256):
        X = rng.uniform(-1.0, 1.0, (n, n))
        spd = X.T @ X + n * np.eye(n)
        gen = rng.uniform(-1.0, 1.0, (n, n)) + n * np.eye(n)
        for A in (spd, gen):
            res = A @ O.inverse_general(A) - np.eye(n)
            assert np.max(np.abs(res)) / max(np.max(np.abs(A)), 1.0) < 1e-11
        ref = np.linalg.solve(gen, np.eye(n))
        assert np.max(np.abs(ref - O.inverse_general(gen))) / np.max(np.abs(ref)) < 1e-11


def schur_S(st, E, n):
    """The matrix sinv_at inverts: A - B D^-1 B^T with the stability shifts."""
    h2_6 = st.dr * st.dr / 6.0
    A = (1.0 + h2_6 * E) * np.eye(st.n_mu) - h2_6 * O.V_at(st, n)
    if n < O.STAB_N_MAX:
        A, _ = O.stability_shift(O.sym(A))
    if n >= st.n_tr:
        return A
    B = O.B_at(st, n)
    S = A - (B * O.dinv_at(st, n)[None, :]) @ B.T
    if n < O.STAB_N_MAX:
        S, _ = O.stability_shift(S)
    return S


def test_sinv_symmetric_inverse(monkeypatch, setup):
    """test_sinv_symmetric_inverse.cpp, at every radial point: the
    dsytrf + dsytri Sinv is exactly symmetric, Sinv S = I to 1e-10, and it
    is within 1e-10 (relative) of the LU inverse symmetrised as 0.5 (M + M^T)."""
    st = setup
    E = 0.9
    for n in range(st.Nr):
        monkeypatch.setattr(O, "BUILD", "mkl")
        new = O.sinv_at(st, E, n)
        monkeypatch.setattr(O, "BUILD", "eigen")
        legacy = O.sinv_at(st, E, n)
        assert np.array_equal(new, new.T)
        assert np.max(np.abs(new @ schur_S(st, E, n) - np.eye(st.n_mu))) < 1e-10
        assert np.max(np.abs(new - legacy)) / np.max(np.abs(legacy)) < 1e-10

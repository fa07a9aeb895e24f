"""The oracle's building blocks against the acceptance checks of the
reference's component tests (thresholds as there):

  src/tests/test_w_inverse_operator.cpp (1) W^-1 from the Schur structure ==
      LU inverse of the assembled W (W built as build_W_unshifted, :74-111),
      (3) W (W^-1 Z) == Z, (4) W^-1 symmetric, (5) past n_transition W^-1 is
      block-diagonal [Sinv, diag(1/D_clamp)];
  src/tests/test_schur_inverter.cpp  Sinv S == I, Sinv symmetric;
  src/tests/test_exchange_coupling.cpp  the CSR exchange coupling == the
      triple loop sum_lambda G(mu, lambda, sigma) chi_{i,lambda}(r).
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

"""The hand-written reverse pass of the Schur + Numerov recurrence
(oracle/adjoint_recurrence.py) against the autograd gradient of
oracle/adjoint.py, for J = sum(C * K) with a random C.

dJ/dV(n) at every grid point, and through it dJ/dalpha and dJ/dr_c, must
agree to rounding.  The checkpointed reverse (one Rinv kept every `segment`
steps, segments recomputed) must give the same bits for any segment length.
"""
import dataclasses

import numpy as np
import pytest
import torch

from oracle import adjoint as AD
from oracle import adjoint_recurrence as AR
from oracle import solver as O
from scatt_b200 import synth

ALPHA, RC, E = 9.6, 1.5, 0.6


def _case(Nr, dr, l_cont, bump_at=None):
    """The H2-like setup, V(n) with V_pol, and optionally a repulsive bump
    3000 I + sym(random) on V(bump_at): above 6 / h^2 it makes A(n)
    indefinite, so the stability shift enters the recurrence there (the
    inputs alone shift only below n_start, where the analytic start is used)."""
    base = dataclasses.replace(synth.h2_like(Nr=Nr, dr=dr, l_cont=l_cont), alpha_pol=0.0, pol_form=1, r_c=RC)
    st = O.make_setup(base)
    bump = np.zeros((Nr, st.n_mu, st.n_mu))
    if bump_at is not None:
        R = np.random.default_rng(2).standard_normal((st.n_mu, st.n_mu))
        bump[bump_at] = 3000.0 * np.eye(st.n_mu) + 50.0 * (R + R.T)

    def dvp_dalpha(n):
        r = n * dr
        return 0.0 if r < 1e-6 else -1.0 / (2.0 * (r * r + RC * RC) ** 2)

    def dvp_drc(n):
        r = n * dr
        return 0.0 if r < 1e-6 else 2.0 * ALPHA * RC / (r * r + RC * RC) ** 3

    def V_of(n):
        return O.V_at(st, n) + ALPHA * dvp_dalpha(n) * np.eye(st.n_mu) + bump[n]

    C = np.random.default_rng(1).standard_normal((st.n_mu, st.n_mu))
    return st, V_of, C, dvp_dalpha, dvp_drc, bump


def _hand_written(st, V_of, C, segment):
    P = AD.Problem(st, pol_form=1)
    rec = AR.Recurrence(st, E, V_of, segment=segment)
    leaf = torch.tensor(rec.Rinv_last, requires_grad=True)       # the small KME stage by autograd
    torch.sum(torch.as_tensor(C) * AD._kme(P, E, leaf, st.Nr - 2)).backward()
    return rec, rec.reverse(leaf.grad.numpy())


@pytest.mark.parametrize("Nr,dr,l_cont,bump_at", [(801, 0.05, 2, None), (401, 0.1, 4, None), (801, 0.05, 2, 20)])
def test_reverse_pass_equals_autograd(Nr, dr, l_cont, bump_at):
    st, V_of, C, dvp_dalpha, dvp_drc, bump = _case(Nr, dr, l_cont, bump_at)
    _, Vbar = _hand_written(st, V_of, C, AR.SEGMENT)
    P = AD.Problem(st, pol_form=1)
    alpha = torch.tensor(ALPHA, dtype=torch.float64, requires_grad=True)
    rc = torch.tensor(RC, dtype=torch.float64, requires_grad=True)
    dV = torch.tensor(bump, dtype=torch.float64, requires_grad=True)
    J = torch.sum(torch.as_tensor(C) * AD.k_matrix(P, E, alpha, rc, dV))
    ga, gr, gV = torch.autograd.grad(J, (alpha, rc, dV))
    gV = gV.numpy()
    assert np.max(np.abs(Vbar - gV)) <= 1e-10 * np.max(np.abs(gV))
    tr = np.einsum("nii->n", Vbar)
    a = sum(tr[n] * dvp_dalpha(n) for n in range(st.Nr))
    r = sum(tr[n] * dvp_drc(n) for n in range(st.Nr))
    assert abs(a - ga.item()) <= 1e-10 * abs(ga.item())
    assert abs(r - gr.item()) <= 1e-10 * abs(gr.item())
    shifted = [n for n in range(O.n_start(st), O.STAB_N_MAX) if AR.Step(st, E, n, V_of(n)).vA is not None]
    assert shifted == ([] if bump_at is None else [bump_at])


def test_segment_length_does_not_change_the_result():
    st, V_of, C, _, _, _ = _case(801, 0.05, 2, bump_at=20)
    ref_rec, ref = _hand_written(st, V_of, C, st.Nr)                     # no intermediate checkpoint
    for seg in (256, 7, 1):
        rec, Vbar = _hand_written(st, V_of, C, seg)
        assert np.array_equal(Vbar, ref)
        assert len(rec.checkpoints) == 1 + (rec.n_last - (rec.ns - 1)) // seg
    assert len(ref_rec.checkpoints) == 1

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


# ------------------------------------------------- the dipoles (back sweep)
def _degenerate_shifts(st, V_of):
    """Grid points where a stability shift is taken while lambda_min of the
    shifted matrix is degenerate (the m = +-l pair of the H2-like system at
    n = 1).  The shift W_min - lambda_min + margin is not differentiable
    there: dJ/dV(n) is undefined, and each method returns the subgradient of
    the eigenvector LAPACK picks.  The derivative along directions that keep
    the degeneracy, c I among them (alpha and r_c act so), is defined."""
    h2_6 = st.dr * st.dr / 6.0
    out = []
    for n in range(O.STAB_N_MAX):
        if AR.Step(st, E, n, V_of(n)).vA is None:          # A shifts are the ones these inputs take
            continue
        A = np.eye(st.n_mu) * (1.0 + h2_6 * E) - h2_6 * V_of(n)
        w = np.linalg.eigvalsh(0.5 * (A + A.T))
        if w[1] - w[0] <= 1e-12 * np.max(np.abs(w)):
            out.append(n)
    return out


def _compare(Vbar, gV, skip):
    """Full comparison except at `skip`, where only the trace is compared."""
    scale = np.max(np.abs(gV))
    keep = np.ones(len(gV), dtype=bool)
    keep[skip] = False
    assert np.max(np.abs(Vbar[keep] - gV[keep])) <= 1e-10 * scale
    for n in skip:
        assert abs(np.trace(Vbar[n]) - np.trace(gV[n])) <= 1e-10 * scale


def _objective(n_mu):
    rng = np.random.default_rng(3)
    Cs = [torch.as_tensor(rng.standard_normal(n_mu) + 1j * rng.standard_normal(n_mu)) for _ in range(6)]
    return lambda Ds: sum(torch.sum(torch.abs(d) ** 2) * (s + 1) + torch.real(torch.sum(Cs[s] * d))
                          for s, d in enumerate(Ds))


@pytest.mark.parametrize("Nr,dr,l_cont", [(801, 0.05, 2), (401, 0.1, 4)])
def test_dipole_forward_and_reverse(Nr, dr, l_cont):
    """Forward: D from the accumulation G(n) equals solve_energy's D.
    Reverse: dJ/dV(n) for every n, and dJ/dalpha, dJ/dr_c, equal autograd.
    (At l_cont = 4 the stability shift at n = 1 enters through psi_1.)"""
    st, V_of, _, dvp_dalpha, dvp_drc, _ = _case(Nr, dr, l_cont)
    da = AR.DipoleAdjoint(st, E, V_of)
    ref = O.solve_energy(O.make_setup(dataclasses.replace(st.inp, alpha_pol=ALPHA)), E)
    for s, D in enumerate(da.dipoles()):
        assert np.max(np.abs(D - ref.slices[s]["D"])) <= 1e-12 * np.max(np.abs(ref.slices[s]["D"]))
    obj = _objective(st.n_mu)
    Vbar = da.reverse(obj)
    P = AD.Problem(st, pol_form=1)
    alpha = torch.tensor(ALPHA, dtype=torch.float64, requires_grad=True)
    rc = torch.tensor(RC, dtype=torch.float64, requires_grad=True)
    dV = torch.zeros(st.Nr, st.n_mu, st.n_mu, dtype=torch.float64, requires_grad=True)
    ga, gr, gV = torch.autograd.grad(obj(AD.dipoles(P, E, alpha, rc, dV)), (alpha, rc, dV))
    gV = gV.numpy()
    skip = _degenerate_shifts(st, V_of)
    assert skip == ([1] if l_cont == 4 else [])
    _compare(Vbar, gV, skip)
    tr = np.einsum("nii->n", Vbar)
    assert abs(sum(tr[n] * dvp_dalpha(n) for n in range(st.Nr)) - ga.item()) <= 1e-10 * abs(ga.item())
    assert abs(sum(tr[n] * dvp_drc(n) for n in range(st.Nr)) - gr.item()) <= 1e-10 * abs(gr.item())


def test_dipole_reverse_segment_length_does_not_change_the_result():
    st, V_of, _, _, _, _ = _case(401, 0.1, 4)
    obj = _objective(st.n_mu)
    ref = AR.DipoleAdjoint(st, E, V_of, segment=st.Nr).reverse(obj)
    for seg in (256, 7, 1):
        assert np.array_equal(AR.DipoleAdjoint(st, E, V_of, segment=seg).reverse(obj), ref)


def test_time_delay_gradient_across_energies():
    """tau couples energies through dD/dE: dJ/dD per energy comes from
    autograd of the small observable stage (delta J = Re sum conj(g) delta D),
    each energy's reverse runs on that linear objective, and the sum over
    energies equals autograd through the whole chain."""
    st, V_of, _, _, _, _ = _case(401, 0.1, 4)
    Es = [0.5, 0.6, 0.72]
    e_homo = float(st.inp.orb_energies[st.n_occ - 1])
    P = AD.Problem(st, pol_form=1)
    alpha = torch.tensor(ALPHA, dtype=torch.float64)
    rc = torch.tensor(RC, dtype=torch.float64)
    dV = torch.zeros(st.Nr, st.n_mu, st.n_mu, dtype=torch.float64, requires_grad=True)
    J = AD.observables(P, Es, e_homo, alpha, rc, dV)["tau_length_z"][1]
    gV, = torch.autograd.grad(J, (dV,))
    # the same by hand: D leaves -> g per energy -> per-energy reverse
    das = [AR.DipoleAdjoint(st, E_, V_of) for E_ in Es]
    leaves = [[torch.tensor(d, requires_grad=True) for d in da.dipoles()] for da in das]
    k = [np.sqrt(2.0 * E_) for E_ in Es]
    D = torch.stack([leaves[e][2] for e in range(len(Es))])            # slot (L, z)
    kk = torch.tensor(k, dtype=torch.float64)
    tau = torch.sum(torch.conj(D) * (AD.d_dk(k, D) / kk[:, None]), dim=1).imag / torch.sum(torch.abs(D) ** 2, dim=1)
    grads = torch.autograd.grad(tau[1], [x for ls in leaves for x in ls], allow_unused=True)
    Vbar = np.zeros_like(gV.numpy())
    for e, da in enumerate(das):
        g = [grads[6 * e + s] if grads[6 * e + s] is not None else torch.zeros(st.n_mu, dtype=torch.complex128)
             for s in range(6)]
        Vbar += da.reverse(lambda Ds, g=g: sum(torch.real(torch.sum(torch.conj(g[s]) * Ds[s])) for s in range(6)))
    _compare(Vbar, gV.numpy(), _degenerate_shifts(st, V_of))

"""The small stages of the device adjoint (scatt_b200.adjoint, run in torch
after the library's sweep) against the oracle's DipoleAdjoint, on the CPU.

The torch stages take the window store (Rinv(n), Sinv(n) for n_s <= n < N),
G(N-1), V(N), B(N) and the dipole rows at N -- here the oracle's own values
-- and must reproduce the oracle's six dipoles; their gradients with respect
to those inputs are what the library's reverse pass consumes.
"""
import dataclasses
import types

import numpy as np
import pytest
import torch

from oracle import adjoint_recurrence as AR
from oracle import solver as O
from scatt_b200 import adjoint as ADJ
from scatt_b200 import synth

E = 0.6


def _inputs(inp):
    st = O.make_setup(inp)
    da = AR.DipoleAdjoint(st, E, lambda n: O.V_at(st, n), segment=64)
    Nr, Np, Nt, Nf = st.Nr, st.n_mu, st.Nt, st.Nf
    N = Nr - 1
    wlo, whi = O.aa_window(st)
    K = 6 + st.n_occ
    v = types.SimpleNamespace(N=N, n_s=wlo, n_window=N - wlo, n_tr=st.n_tr, n_pts=da.n_hi, ne_fit=whi, Np=Np,
                              Nt=Nt, Nf=Nf, Krows=K, Np_max=Np, E=E)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64)
    Rraw = t(np.stack([da.window[m][0].T for m in range(wlo, N)]))
    Sraw = t(np.stack([da.window[m][1].Sinv.T for m in range(wlo, N)]))
    BN = O.B_at(st, N)
    arrays = {"Rraw": Rraw, "Sraw": Sraw, "Graw": t(da.G_last), "VN": t(O.V_at(st, N)),
              "BN": t(BN) if Nf else None, "BsN": t(BN * O.dinv_at(st, N)[None, :]) if Nf else None,
              "CN": t(da.L[N].T) if N < da.n_hi else None}
    if Nf and any(m < st.n_tr for m in range(wlo, N)):
        arrays["Bsw"] = t(np.stack([(O.B_at(st, m) * O.dinv_at(st, m)[None, :]).T for m in range(wlo, N)]))
    d_corr = np.array([[O.simpson((st.dr + np.arange(da.n_hi) * st.dr if s < 3 else np.ones(da.n_hi))
                                  * np.sum(st.phi[a, :da.n_hi, :min(Np, st.n_lambda)]
                                           * O.xi_tables(st, 0, da.n_hi)[s][:, :min(Np, st.n_lambda)], axis=1), st.dr)
                        for a in range(st.n_occ)] for s in range(6)])
    en = ADJ._Energy(v, st.dr, torch.device("cpu"), 1, d_corr, st.spin, arrays=arrays)
    return st, da, en


@pytest.mark.parametrize("builder,kw", [
    ("h2_like", dict(Nr=401, dr=0.1, l_cont=4)),
    ("h2o_like", dict(Nr=301, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)),
])
def test_small_stages_reproduce_the_oracle_dipoles(builder, kw):
    st, da, en = _inputs(getattr(synth, builder)(**kw))
    D = en.dipoles()
    ref = da.dipoles()
    for s in range(6):
        # reordered sums (torch vs numpy contractions over the window) only
        assert np.max(np.abs(D[s].detach().numpy() - ref[s])) <= 1e-10 * np.max(np.abs(ref[s]))
    np.testing.assert_allclose(en.A.detach().numpy(), da.A, rtol=0, atol=1e-10 * np.max(np.abs(da.A)))


def test_small_stage_gradients_match_finite_differences():
    """dJ/dG(N-1), dJ/dRinv and dJ/dSinv over the window from autograd of the
    torch stages, against central differences of the same stages."""
    st, da, en = _inputs(synth.h2_like(Nr=401, dr=0.1, l_cont=3))
    w = [torch.as_tensor(np.random.default_rng(s).standard_normal(st.n_mu)) for s in range(6)]
    J = lambda Ds: sum(torch.sum(w[s] * torch.abs(Ds[s]) ** 2) for s in range(6))
    J(en.dipoles()).backward()
    # Rinv(N - 1) enters through its inverse, which is far from linear: a smaller step
    grads = [(leaf, leaf.grad.clone(), rel) for leaf, rel in ((en.Graw, 1e-6), (en.Rraw, 1e-8), (en.Sraw, 1e-6))]
    rng = np.random.default_rng(9)
    for leaf, g, rel in grads:
        d = torch.as_tensor(rng.standard_normal(tuple(leaf.shape)))
        h = rel * float(torch.max(torch.abs(leaf)))
        with torch.no_grad():
            leaf += h * d
            jp = float(J(en.dipoles()))
            leaf -= 2 * h * d
            jm = float(J(en.dipoles()))
            leaf += h * d
        fd = (jp - jm) / (2 * h)
        an = float(torch.sum(g * d))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-30)

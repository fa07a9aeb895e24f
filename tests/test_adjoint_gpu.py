"""Device adjoint (scatt_adjoint_*, scatt_b200.adjoint) against the oracle's
hand-written DipoleAdjoint and against central finite differences.

* dJ/dV(n) at every grid point (summed over the energies, and its trace per
  energy) equals the oracle's to 1e-8 of its largest entry.  Where a
  stability shift is taken at a degenerate lambda_min only the trace is
  compared: the shift is not differentiable there and the library averages
  over the degenerate eigenvectors while LAPACK picks one.
* The checkpoint segment length does not change the result.
* d sigma / d alpha, d sigma / d r_c and d tau / d alpha agree with central
  differences (h = 1e-6 relative) to 1e-6; dJ/dV_ll'(r) at single grid
  entries agrees to 1e-6 with Richardson-extrapolated central differences
  at h = 1e-4 (at 1e-6 the solve's rounding noise dominates a single
  entry's difference quotient).
"""
import dataclasses

import numpy as np
import pytest
import torch

from oracle import adjoint_recurrence as AR
from oracle import solver as O
from scatt_b200 import adjoint as ADJ
from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu

ALPHA, RC, E = 9.6, 1.5, 0.6
CASES = [("h2o_like", dict(Nr=301, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)),
         ("h2_like", dict(Nr=401, dr=0.1, l_cont=4))]


def _case(builder, kw):
    inp = dataclasses.replace(getattr(synth, builder)(**kw), alpha_pol=ALPHA, pol_form=1, r_c=RC)
    st = O.make_setup(dataclasses.replace(inp, alpha_pol=0.0))

    def vp(n):
        r = n * st.dr
        return 0.0 if r < 1e-6 else -ALPHA / (2.0 * (r * r + RC * RC) ** 2)

    return inp, st, (lambda n: O.V_at(st, n) + vp(n) * np.eye(st.n_mu))


def _objective(n_mu):
    rng = np.random.default_rng(3)
    Cs = [rng.standard_normal(n_mu) + 1j * rng.standard_normal(n_mu) for _ in range(6)]
    return lambda Ds: sum(torch.sum(torch.abs(d) ** 2) * (s + 1)
                          + torch.real(torch.sum(torch.as_tensor(Cs[s], device=d.device) * d))
                          for s, d in enumerate(Ds))


def _degenerate_shifts(st, V_of):
    h2_6 = st.dr * st.dr / 6.0
    out = []
    for n in range(O.STAB_N_MAX):
        if AR.Step(st, E, n, V_of(n)).vA is None:
            continue
        A = np.eye(st.n_mu) * (1.0 + h2_6 * E) - h2_6 * V_of(n)
        w = np.linalg.eigvalsh(0.5 * (A + A.T))
        if w[1] - w[0] <= 1e-12 * np.max(np.abs(w)):
            out.append(n)
    return out


@pytest.mark.parametrize("builder,kw", CASES)
def test_device_adjoint_equals_oracle(builder, kw):
    inp, st, V_of = _case(builder, kw)
    sol = S.ScanSolver(inp)
    adj = ADJ.ScanAdjoint(sol, [E], segment=64)
    Ds = adj.dipoles()[0]
    da = AR.DipoleAdjoint(st, E, V_of)
    ref = da.dipoles()
    for s in range(6):
        assert np.max(np.abs(Ds[s].detach().cpu().numpy() - ref[s])) <= 1e-10 * np.max(np.abs(ref[s]))
    J = _objective(st.n_mu)
    J(list(Ds)).backward()
    vtr, vfull = adj.reverse(full=True)
    Vbar = da.reverse(J)
    Vd = vfull.transpose(1, 2).cpu().numpy()[:, :st.n_mu, :st.n_mu]
    scale = np.max(np.abs(Vbar))
    skip = _degenerate_shifts(st, V_of)
    keep = np.ones(st.Nr, dtype=bool)
    keep[skip] = False
    assert np.max(np.abs(Vd[keep] - Vbar[keep])) <= 1e-8 * scale
    tr = np.einsum("nii->n", Vbar)
    assert np.max(np.abs(vtr[0] - tr)) <= 1e-8 * scale
    assert np.max(np.abs(np.einsum("nii->n", Vd) - tr)) <= 1e-8 * scale


def test_segment_length_does_not_change_the_gradient():
    inp, st, _ = _case(*CASES[1])
    sol = S.ScanSolver(inp)
    J = _objective(st.n_mu)
    out = []
    for seg in (8, 64, 512):
        adj = ADJ.ScanAdjoint(sol, [E, 0.9], segment=seg)
        Ds = adj.dipoles()
        (J(list(Ds[0])) + J(list(Ds[1]))).backward()
        out.append(adj.reverse()[0])
        adj.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[1], out[2])


def test_adjoint_forward_equals_the_solver():
    inp, st, _ = _case(*CASES[0])
    sol = S.ScanSolver(inp)
    Es = [0.4, 0.6, 0.9]
    ref = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1))
    adj = ADJ.ScanAdjoint(sol, Es, segment=32)
    for r, a, D in zip(ref, adj.results, adj.dipoles()):
        for f in ("K_kme", "A", "B", "D", "d_raw", "partial_sigma"):
            assert np.array_equal(getattr(a, f), getattr(r, f)), f
        Dn = D.detach().cpu().numpy()
        assert np.max(np.abs(Dn - r.D)) <= 1e-11 * np.max(np.abs(r.D))


def _objective_obs(sol, Es, e_homo, alpha, r_c, dV=None):
    D = ADJ.Dipoles.apply(alpha, r_c, dV, sol, Es, 1, 64)
    obs = ADJ.observables(Es, D, e_homo)
    return obs["sigma_length_z"][0] + 3.0 * obs["sigma_velocity_x"][2] + 1e-3 * obs["tau_length_z"][1]


def test_parameter_gradients_match_central_differences():
    inp, st, _ = _case(*CASES[0])
    sol = S.ScanSolver(inp)
    Es = [0.5, 0.6, 0.72]
    e_homo = float(inp.orb_energies[inp.n_occ - 1])
    a = torch.tensor(ALPHA, dtype=torch.float64, requires_grad=True)
    rc = torch.tensor(RC, dtype=torch.float64, requires_grad=True)
    J = _objective_obs(sol, Es, e_homo, a, rc)
    J.backward()
    for which, g in (("alpha", a.grad.item()), ("r_c", rc.grad.item())):
        x0 = ALPHA if which == "alpha" else RC
        h = 1e-6 * x0
        vals = []
        for sgn in (1, -1):
            aa = torch.tensor(ALPHA + (sgn * h if which == "alpha" else 0.0), dtype=torch.float64)
            rr = torch.tensor(RC + (sgn * h if which == "r_c" else 0.0), dtype=torch.float64)
            with torch.no_grad():
                vals.append(float(_objective_obs(sol, Es, e_homo, aa, rr)))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - g) <= 1e-6 * abs(g), (which, fd, g)


def test_potential_gradient_matches_central_differences():
    inp, st, _ = _case(*CASES[0])
    sol = S.ScanSolver(inp)
    Es = [0.5, 0.6, 0.72]
    e_homo = float(inp.orb_energies[inp.n_occ - 1])
    Npm = sol.Np
    a = torch.tensor(ALPHA, dtype=torch.float64)
    rc = torch.tensor(RC, dtype=torch.float64)
    dV = torch.zeros((st.Nr, Npm, Npm), dtype=torch.float64, device="cuda", requires_grad=True)
    J0 = _objective_obs(sol, Es, e_homo, a, rc, dV)
    J0.backward()
    J0 = abs(float(J0))
    g = dV.grad
    gmax = float(g.abs().max())
    # the entries with the largest gradients at a few radii, and a few fixed ones
    picks = [(5, 0, 0), (40, 1, 3), (st.Nr - 1, 3, 1)]
    for n in (60, 150, st.Nr - 2):
        flat = int(torch.argmax(g[n].abs()))
        picks.append((n, flat // Npm, flat % Npm))
    def quotient(n, i, j, h):
        vals = []
        for sgn in (1, -1):
            d = torch.zeros((st.Nr, Npm, Npm), dtype=torch.float64, device="cuda")
            d[n, i, j] += sgn * h
            if i != j:
                d[n, j, i] += sgn * h
            with torch.no_grad():
                vals.append(float(_objective_obs(sol, Es, e_homo, a, rc, d)))
        return (vals[0] - vals[1]) / (2 * h)

    for n, i, j in picks:
        # the solve's rounding noise (about 1e-12 |J|) swamps differences of a
        # single grid entry at 1e-6; at 1e-4 with Richardson extrapolation the
        # truncation error is O(h^4)
        h = 1e-4 * max(1.0, float(np.max(np.abs(O.V_at(st, n)))))
        # Richardson: the h^2 term of the central difference cancels
        fd = (4.0 * quotient(n, i, j, 0.5 * h) - quotient(n, i, j, h)) / 3.0
        an = float(g[n, i, j] + (g[n, j, i] if i != j else 0.0))
        # 1e-6 of the entry, plus 1e-7 of the largest gradient entry (the
        # rounding that an ill-conditioned solve carries into small entries),
        # plus the quotient's rounding noise (about 1e-15 |J| over the step)
        noise = 1e-15 * J0 / h
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-7 * gmax + noise, (n, i, j, fd, an, noise)

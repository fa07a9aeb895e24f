"""The gradient checker for the adjoint (oracle/adjoint.py) against central
finite differences of the numpy oracle.

Objectives: sigma_L, sigma_V per polarisation and tau at the middle of three
energies; parameters: alpha and r_c of V_pol = -alpha / (2 (r^2 + r_c^2)^2)
(alpha = 9.6, r_c = 1.5) and V_ll'(r) along a random symmetric direction.

The steps are where central differences of this solver are accurate.  At
h = 1e-6 they are limited by the oracle's own rounding noise, about
1e-12 |J| / h.  That puts them within 1e-8 to 2e-6 (relative) of the exact
derivative for sigma and 6e-6 to 1e-4 for tau, because tau differences
dipoles across energies.  At the steps used here (1e-3 for alpha, which
enters V linearly, 1e-4 otherwise) they agree to 1e-7, and to 3e-7 through
the stability shift.
"""
import dataclasses
import math

import numpy as np
import pytest
import torch

from oracle import adjoint as AD
from oracle import observables as OBS
from oracle import solver as O
from scatt_b200 import synth

ES = [0.5, 0.6, 0.72]
ALPHA, RC = 9.6, 1.5
KEYS = ["sigma_length_z", "sigma_velocity_x", "sigma_velocity_y", "tau_length_z", "tau_velocity_x"]


def oracle_observables(inp, Es, e_homo, perturb=None):
    """sigma and tau of the numpy oracle; perturb(n) is added to V(n)."""
    st = O.make_setup(inp)
    V_orig = O.V_at
    if perturb is not None:
        O.V_at = lambda s, n: V_orig(s, n) + perturb(n)
    try:
        res = [O.solve_energy(st, E) for E in Es]
    finally:
        O.V_at = V_orig
    k = [math.sqrt(2.0 * E) for E in Es]
    om = [E - e_homo for E in Es]
    out = {}
    for s, (g, q) in enumerate(O.SLOTS):
        gauge = "length" if g == "L" else "velocity"
        pol = "xyz"[s % 3]
        D = [list(r.slices[s]["D"]) for r in res]
        out[f"sigma_{gauge}_{pol}"] = np.array(OBS.cross_section(k, D, om, gauge))
        if len(Es) > 1:
            out[f"tau_{gauge}_{pol}"] = np.array(OBS.time_delay(k, D))
    return out, [r.shifts for r in res]


@pytest.fixture(scope="module")
def case():
    base = dataclasses.replace(synth.h2_like(Nr=801, dr=0.05, l_cont=2), alpha_pol=ALPHA, pol_form=1, r_c=RC)
    e_homo = float(base.orb_energies[base.n_occ - 1])
    P = AD.Problem(O.make_setup(dataclasses.replace(base, alpha_pol=0.0)), pol_form=1)
    alpha = torch.tensor(ALPHA, dtype=torch.float64, requires_grad=True)
    rc = torch.tensor(RC, dtype=torch.float64, requires_grad=True)
    dV = torch.zeros(base.Nr, P.st.n_mu, P.st.n_mu, dtype=torch.float64, requires_grad=True)
    obs = AD.observables(P, ES, e_homo, alpha, rc, dV)
    grads = {key: torch.autograd.grad(obs[key][1], (alpha, rc, dV), retain_graph=True) for key in KEYS}
    return base, e_homo, obs, grads


def test_forward_equals_oracle(case):
    base, e_homo, obs, _ = case
    ref, _ = oracle_observables(base, ES, e_homo)
    for key, v in ref.items():
        assert np.max(np.abs(obs[key].detach().numpy() - v) / np.abs(v)) < 1e-12, key


@pytest.mark.parametrize("which", ["alpha", "r_c"])
def test_polarisation_parameter_gradients(case, which):
    base, e_homo, _, grads = case
    # alpha enters V linearly; r_c through 1 / (r^2 + r_c^2)^2, so a smaller step
    h = {"alpha": 1e-3, "r_c": 1e-4}[which]
    shift = {"alpha": (h, 0.0), "r_c": (0.0, h)}[which]
    plus, _ = oracle_observables(dataclasses.replace(base, alpha_pol=ALPHA + shift[0], r_c=RC + shift[1]), ES, e_homo)
    minus, _ = oracle_observables(dataclasses.replace(base, alpha_pol=ALPHA - shift[0], r_c=RC - shift[1]), ES, e_homo)
    for key in KEYS:
        fd = (plus[key][1] - minus[key][1]) / (2.0 * h)
        g = grads[key][0 if which == "alpha" else 1].item()
        assert abs(g - fd) <= 1e-6 * abs(fd), (key, g, fd)


def test_potential_gradient_along_a_direction(case):
    base, e_homo, _, grads = case
    st_nr, n_mu = base.Nr, grads[KEYS[0]][2].shape[1]
    rng = np.random.default_rng(7)
    Pd = rng.standard_normal((st_nr, n_mu, n_mu))
    Pd = 0.5 * (Pd + Pd.transpose(0, 2, 1)) * np.exp(-np.arange(st_nr) * base.dr / 5.0)[:, None, None]
    eps = 1e-4
    plus, _ = oracle_observables(base, ES, e_homo, lambda n: eps * Pd[n])
    minus, _ = oracle_observables(base, ES, e_homo, lambda n: -eps * Pd[n])
    for key in KEYS:
        fd = (plus[key][1] - minus[key][1]) / (2.0 * eps)
        dd = float(torch.sum(grads[key][2] * torch.as_tensor(Pd)))
        assert abs(dd - fd) <= 1e-6 * abs(fd), (key, dd, fd)


def test_gradients_through_a_stability_shift():
    # l_cont = 4 at dr = 0.1: V near the origin makes A indefinite at n = 1
    base = dataclasses.replace(synth.h2_like(Nr=401, dr=0.1, l_cont=4), alpha_pol=ALPHA, pol_form=1, r_c=RC)
    e_homo = float(base.orb_energies[base.n_occ - 1])
    E = [0.6]
    P = AD.Problem(O.make_setup(dataclasses.replace(base, alpha_pol=0.0)), pol_form=1)
    alpha = torch.tensor(ALPHA, dtype=torch.float64, requires_grad=True)
    rc = torch.tensor(RC, dtype=torch.float64, requires_grad=True)
    dV = torch.zeros(base.Nr, P.st.n_mu, P.st.n_mu, dtype=torch.float64, requires_grad=True)
    J = AD.observables(P, E, e_homo, alpha, rc, dV)["sigma_length_z"][0]
    ga, gr, gV = torch.autograd.grad(J, (alpha, rc, dV))
    rng = np.random.default_rng(8)
    Pd = rng.standard_normal((base.Nr, P.st.n_mu, P.st.n_mu))
    Pd = 0.5 * (Pd + Pd.transpose(0, 2, 1))
    Pd[O.STAB_N_MAX:] = 0.0
    # the shift at n = 1 has a degenerate lambda_min (the m = +-l pair), where
    # the shift is not differentiable; along c I (how alpha and r_c act) it is
    Pd[1] = 0.7 * np.eye(P.st.n_mu)
    h = 1e-4
    checks = [
        (ga.item(), dataclasses.replace(base, alpha_pol=ALPHA + h), dataclasses.replace(base, alpha_pol=ALPHA - h), None),
        (gr.item(), dataclasses.replace(base, r_c=RC + h), dataclasses.replace(base, r_c=RC - h), None),
        (float(torch.sum(gV * torch.as_tensor(Pd))), base, base, Pd),
    ]
    for g, inp_p, inp_m, direction in checks:
        pp = (lambda n: h * direction[n]) if direction is not None else None
        pm = (lambda n: -h * direction[n]) if direction is not None else None
        plus, sh_p = oracle_observables(inp_p, E, e_homo, pp)
        minus, sh_m = oracle_observables(inp_m, E, e_homo, pm)
        assert sh_p[0]["A"] >= 1 and sh_p == sh_m
        fd = (plus["sigma_length_z"][0] - minus["sigma_length_z"][0]) / (2.0 * h)
        assert abs(g - fd) <= 1e-6 * abs(fd), (g, fd)

"""The scan observables in torch (scatt_b200.adjoint.observables: on the
dipoles' device and inside the autograd graph) equal the numpy ones
(scatt_b200.observables.scan_observables, pinned to the reference's
post-processing module by tests/test_observables.py), and their gradients
match central differences.  CPU only: torch tensors on the host."""
import types

import numpy as np
import pytest
import torch

from scatt_b200 import adjoint as ADJ
from scatt_b200 import observables as OB


def _dipoles(nE=6, Np=9, seed=4):
    rng = np.random.default_rng(seed)
    E = np.sort(rng.uniform(0.2, 1.5, nE))
    D = rng.standard_normal((nE, 6, Np)) + 1j * rng.standard_normal((nE, 6, Np))
    return E, D


def test_torch_observables_equal_numpy():
    E, D = _dipoles()
    e_homo = -0.5
    ref = OB.scan_observables([types.SimpleNamespace(E=e, D=d) for e, d in zip(E, D)], e_homo)
    Dt = torch.view_as_real(torch.tensor(D))                     # (nE, 6, Np, 2)
    got = ADJ.observables(E, Dt, e_homo)
    for key in [k for k in ref if k not in ("E", "k", "omega")]:
        assert key in got, key
        np.testing.assert_allclose(got[key].numpy(), ref[key], rtol=1e-12, atol=1e-14, err_msg=key)


@pytest.mark.parametrize("key", ["beta_length", "q_z", "dphi_rms_x", "tau_velocity_y"])
def test_torch_observable_gradients(key):
    E, D = _dipoles(nE=4, Np=4, seed=8)
    Dt = torch.view_as_real(torch.tensor(D)).clone().requires_grad_(True)
    f = lambda X: ADJ.observables(E, X, -0.5)[key].sum()
    f(Dt).backward()
    g = Dt.grad.clone()
    h = 1e-6
    rng = np.random.default_rng(0)
    for _ in range(6):
        idx = tuple(int(rng.integers(0, n)) for n in Dt.shape)
        Xp, Xm = Dt.detach().clone(), Dt.detach().clone()
        Xp[idx] += h
        Xm[idx] -= h
        fd = (f(Xp) - f(Xm)).item() / (2 * h)
        assert abs(g[idx].item() - fd) <= 1e-6 * max(1.0, abs(fd)), (key, idx)

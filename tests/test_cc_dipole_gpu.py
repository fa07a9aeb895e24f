"""The device continuum-continuum dipole (scatt_cc_dipole, the consumer of
the psi store: postprocessing/two_photon_delay/cc_dipole/src/CCDipole.cpp)
against the oracle's restatement of CCDipole.cpp on the same psi, and the
reference's own acceptance checks of it
(postprocessing/two_photon_delay/cc_dipole/tests/): cc(kappa, kappa)
symmetric, cc(kappa, nu) = cc(nu, kappa)^T.  psi comes from the device psi
sweep (held to the oracle's back-propagation in test_psi_gpu.py), so the
comparison isolates the consumer: same inputs, different summation order,
1e-12 relative."""
import numpy as np
import pytest

from oracle import cc_dipole as CC
from scatt_b200 import _lib
from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def states():
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=2)
    sol = S.ScanSolver(inp, device=0)
    keep_hi = min(inp.Nr - 1, max(1, sol.n_transition - 1))
    _, psi = sol.psi_sweep([0.5, 0.7], n_lo=0, n_hi=keep_hi + 1, segment=32,
                           opts=S.default_opts(allow_closed_channels=1))
    sol.close()
    return inp, np.array(psi), keep_hi


@pytest.mark.parametrize("pol", ["x", "y", "z"])
def test_cc_dipole_matches_oracle(states, pol):
    inp, psi, keep_hi = states
    n_mu = psi.shape[-1]
    got = _lib.cc_dipole(psi[0], psi, 0, inp.dr, pol)           # kappa = E 0.5 against both
    for v in range(2):
        ref = CC.cc_dipole(inp.dr, inp.Nr, {n: psi[0, n] for n in range(keep_hi + 1)},
                           {n: psi[v, n] for n in range(keep_hi + 1)}, (0, keep_hi), (0, keep_hi), pol)
        assert got[v].shape == (n_mu, n_mu)
        assert rel(got[v], ref) <= 1e-12, (pol, v)
    # test_cc_dipole_symmetry.cpp: cc(kappa, kappa) is symmetric
    assert np.max(np.abs(got[0] - got[0].T)) <= 1e-12 * np.max(np.abs(got[0]))
    # test_cc_dipole_two_energy.cpp: cc(kappa, nu) = cc(nu, kappa)^T
    back = _lib.cc_dipole(psi[1], psi[0], 0, inp.dr, pol)[0]
    assert rel(back.T, got[1]) <= 1e-12


def test_cc_dipole_even_window_and_chunks(states):
    """An even number of points (the 3/8 tail of CCDipole.cpp:100-122) and a
    window that starts inside the grid."""
    inp, psi, keep_hi = states
    lo, hi = 7, keep_hi + 1 if (keep_hi + 1 - 7) % 2 == 0 else keep_hi
    got = _lib.cc_dipole(psi[1, lo:hi], psi[0, lo:hi], lo, inp.dr, "z")[0]
    ref = CC.cc_dipole(inp.dr, inp.Nr, {n: psi[1, n] for n in range(lo, hi)},
                       {n: psi[0, n] for n in range(lo, hi)}, (lo, hi - 1), (lo, hi - 1), "z")
    assert (hi - lo) % 2 == 0
    assert rel(got, ref) <= 1e-12


def test_cc_dipole_rejects_short_windows(states):
    _, psi, _ = states
    with pytest.raises(_lib.ScattError):
        _lib.cc_dipole(psi[0, :4], psi[1, :4], 0, 0.05, "x")

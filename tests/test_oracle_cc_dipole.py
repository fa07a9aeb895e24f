"""The oracle's continuum-continuum dipole (oracle/cc_dipole.py) against the
acceptance checks of the reference's own tests of it
(postprocessing/two_photon_delay/cc_dipole/tests/):

  test_cc_dipole_symmetry.cpp   cc(kappa, kappa) symmetric (1e-14 abs, 1e-12 rel);
  test_cc_dipole_two_energy.cpp cc(kappa, nu) = cc(nu, kappa)^T at two energies;
  test_cc_dipole_bruteforce.cpp the per-point contraction against an explicit
                                sum over (mu, nu) and the radial points.

The H2O fixture is replaced by the synthetic H2-like system.  The Simpson
weights equal the dipole module's for every window of 5 or more points.
"""
import numpy as np
import pytest

from oracle import cc_dipole as CC
from oracle import solver as O
from scatt_b200 import synth


@pytest.fixture(scope="module")
def states():
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=2)
    st = O.make_setup(inp)
    out = {}
    for E in (0.5, 0.7):
        r = O.solve_energy(st, E, keep_psi=True)
        keep_hi = min(st.Nr - 1, max(1, st.n_tr - 1))
        out[E] = ({n: p for n, p in r.psi_keep.items() if n <= keep_hi}, (0, keep_hi))
    return st, out


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("pol", ["x", "y", "z"])
def test_same_energy_symmetry(states, pol):
    st, s = states
    psi, keep = s[0.5]
    cc = CC.cc_dipole(st.dr, st.Nr, psi, psi, keep, keep, pol)
    assert np.max(np.abs(cc - cc.T)) <= max(1e-14, 1e-12 * np.max(np.abs(cc)))
    assert np.max(np.abs(cc)) > 0.0


@pytest.mark.parametrize("pol", ["x", "y", "z"])
def test_two_energy_transpose(states, pol):
    st, s = states
    (pk, kk), (pn, kn) = s[0.5], s[0.7]
    a = CC.cc_dipole(st.dr, st.Nr, pk, pn, kk, kn, pol)
    b = CC.cc_dipole(st.dr, st.Nr, pn, pk, kn, kk, pol)
    assert np.max(np.abs(a - b.T)) <= max(1e-14, 1e-12 * np.max(np.abs(a)))


def test_bruteforce_sum(states):
    st, s = states
    (pk, kk), (pn, kn) = s[0.5], s[0.7]
    n_lo, n_hi = CC.window(st.Nr, kk, kn, n_overlap_hi=60)
    w = CC.simpson_weights(n_hi - n_lo, st.dr)
    A = CC.ang_table(st.n_mu, CC.Q_OF["z"])
    ref = np.zeros((st.n_mu, st.n_mu))
    for ir in range(n_lo, n_hi):
        r = st.dr + ir * st.dr
        for b in range(st.n_mu):
            for a in range(st.n_mu):
                ref[b, a] += w[ir - n_lo] * r * sum(pk[ir][mu, b] * A[mu, nu] * pn[ir][nu, a]
                                                    for mu in range(st.n_mu) for nu in range(st.n_mu))
    got = CC.cc_dipole(st.dr, st.Nr, pk, pn, kk, kn, "z", n_overlap_hi=60)
    assert _rel(got, ref) < 1e-12


def test_weights_and_limits(states):
    st, s = states
    for n in range(5, 40):
        w = CC.simpson_weights(n, 0.1)
        f = np.random.default_rng(n).standard_normal(n)
        assert abs(w @ f - O.simpson(f, 0.1)) <= 1e-14 * np.sum(np.abs(f))
    psi, keep = s[0.5]
    with pytest.raises(RuntimeError, match="only length gauge"):
        CC.cc_dipole(st.dr, st.Nr, psi, psi, keep, keep, "z", gauge="velocity")
    with pytest.raises(RuntimeError, match="too few overlapping"):
        CC.window(st.Nr, (0, 3), (0, 100))

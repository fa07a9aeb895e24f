"""How far rounding alone moves the path's observables (CPU oracle).

The Numerov R-ratio recurrence with closed channels amplifies rounding: on
the H2O-like case of the solver tests (l_cont 11, two orbitals, N_t = 386,
301 points at dr = 0.05, E = 0.3), additive noise of 1e-16 x max|Rinv(n)|
on every entry of every R-ratio inverse -- the size of one rounding error
per entry -- moves K by about 1e-8 and the dipoles by about 1e-9 (relative
to their largest entries).  Any two correct FP64 implementations that round
differently (LU vs Gauss-Jordan, 64- vs 128-column windows, back sweep vs
forward accumulation) therefore differ by that much on such a case, which is
why the GPU parity tolerances are set against each case's measured floor
rather than a fixed 1e-10.
"""
import numpy as np

from oracle import solver as O
from scatt_b200 import synth


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_rounding_noise_moves_k_and_dipoles_above_1e_10(monkeypatch):
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=11, lmax_orb=8, n_orb=2)
    st = O.make_setup(inp)
    E = 0.3
    r0 = O.solve_energy(st, E)
    rng = np.random.default_rng(1)
    frp = O.frp_step

    def noisy(st_, n, Sinv, prev):
        X = frp(st_, n, Sinv, prev)
        N = rng.standard_normal(X.shape) * 1e-16
        return X + 0.5 * (N + N.T) * np.max(np.abs(X))

    monkeypatch.setattr(O, "frp_step", noisy)
    r1 = O.solve_energy(st, E)
    dK = _rel(r1.K_kme, r0.K_kme)
    dD = max(_rel(r1.slices[s]["D"], r0.slices[s]["D"]) for s in range(6))
    assert 1e-9 < dK < 1e-6, dK
    assert 1e-10 < dD < 1e-7, dD

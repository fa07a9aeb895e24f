"""Cross sections and Wigner delays of a scan (host arithmetic on the solver's
dipoles) against the oracle's loop restatement and an analytic phase."""
import numpy as np

from oracle import observables as OO
from scatt_b200 import observables as OBS


def _dipoles(k, nc=5, seed=3):
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.5, 2.0, nc)
    phase0 = rng.uniform(-1, 1, nc)
    slope = rng.uniform(-2, 2, nc)
    # smooth amplitude and phase per channel
    return (amp[None, :] * (1 + 0.1 * k[:, None]) *
            np.exp(1j * (phase0[None, :] + slope[None, :] * k[:, None] ** 2)))


def test_matches_oracle_on_uneven_grid():
    k = np.sort(np.random.default_rng(1).uniform(0.1, 2.0, 23))
    D = _dipoles(k)
    om = 0.5 * k ** 2 + 0.46
    for g in ("length", "velocity"):
        a = OBS.cross_section(k, D, om, g)
        b = np.array(OO.cross_section(list(k), [list(r) for r in D], list(om), g))
        assert np.allclose(a, b, rtol=1e-14, atol=0)
    a = OBS.time_delay(k, D)
    b = np.array(OO.time_delay(list(k), [list(r) for r in D]))
    assert np.allclose(a, b, rtol=1e-12, atol=1e-14)
    assert np.allclose(OBS.time_delay(k, D, with_minus=True), -a)


def test_delay_of_a_known_phase():
    # one channel, phase s k^2: d(phase)/dE = (2 s k) / k = 2 s exactly; the
    # central difference of exp(i s k^2) errs by ~ h^2 (2 s k)^2 / 6 relative
    k = np.linspace(0.2, 2.0, 400)
    h = k[1] - k[0]
    D = (1.3 * np.exp(1j * 0.7 * k ** 2))[:, None]
    tau = OBS.time_delay(k, D)
    bound = 1.4 * h * h * (1.4 * k[1:-1]) ** 2 / 6 * 1.5
    assert np.all(np.abs(tau[1:-1] - 1.4) < bound)


def test_gauge_ratio_is_one_when_dv_equals_omega_dl():
    k = np.linspace(0.3, 1.5, 9)
    om = 0.5 * k ** 2 + 0.5
    DL = _dipoles(k)
    DV = om[:, None] * DL
    assert np.allclose(OBS.q_sigma(DL, DV, om), 1.0, rtol=1e-13)
    assert np.allclose(OBS.cross_section(k, DL, om, "length"), OBS.cross_section(k, DV, om, "velocity"),
                       rtol=1e-13)

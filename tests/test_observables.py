"""Scan observables (host arithmetic on the solver's dipoles): cross
sections, Wigner delays, the gauge ratio and phase spread, and the asymmetry
parameter beta, against the oracle's loop restatement, an analytic phase,
the beta limits and a closed form of beta in real Gaunt coefficients."""
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


def _three_pols(n_e=2, l_max=3, seed=5):
    rng = np.random.default_rng(seed)
    n = (l_max + 1) ** 2
    return [rng.standard_normal((n_e, n)) + 1j * rng.standard_normal((n_e, n)) for _ in range(3)]


def test_dphi_rms_and_beta_match_the_oracle():
    DL, DV, _ = _three_pols(3, 3, seed=6)
    assert np.allclose(OBS.dphi_rms(DL, DV), OO.dphi_rms([list(r) for r in DL], [list(r) for r in DV]),
                       rtol=1e-13, atol=0)
    D = _three_pols(2, 2)
    got = OBS.beta(*D, n_theta=12, n_phi=24)
    ref = OO.beta(*[[list(r) for r in d] for d in D], n_theta=12, n_phi=24)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-13)


def test_beta_limits():
    # atomic s -> p: D^(q) on the l = 1 channel along q gives beta = 2
    D = [np.zeros((1, 4), complex) for _ in range(3)]
    D[0][0, 3] = D[1][0, 1] = D[2][0, 2] = 0.7 - 0.2j          # (1, +1) = x, (1, -1) = y, (1, 0) = z
    assert abs(OBS.beta(*D)[0] - 2.0) < 1e-13
    # D^(q)(k) = (k x a)_q has no component along k: N_1 = 0, beta = -1
    ax, ay, az = 0.3, -1.1, 0.8 + 0.4j
    X, Y, Z = 3, 1, 2                                           # l = 1 channels along x, y, z
    D = [np.zeros((1, 4), complex) for _ in range(3)]
    D[0][0, Y], D[0][0, Z] = az, -ay                           # k_y a_z - k_z a_y
    D[1][0, Z], D[1][0, X] = ax, -az                           # k_z a_x - k_x a_z
    D[2][0, X], D[2][0, Y] = ay, -ax                           # k_x a_y - k_y a_x
    assert abs(OBS.beta(*D)[0] + 1.0) < 1e-13
    # and any amplitudes stay within [-1, 2]
    b = OBS.beta(*_three_pols(50, 6, seed=7))
    assert np.all(b >= -1.0 - 1e-12) and np.all(b <= 2.0 + 1e-12)


def test_beta_quadrature_is_exact_below_its_degree():
    """N_1 = (4 pi / 3) sum_lambda |sum_{q, mu} d^(q)_mu G(mu; 1 q; lambda)|^2 in
    real Gaunt coefficients and sigma_tot = 1/3 sum |d|^2 (orthonormality):
    the default 40 x 80 grid reproduces this closed form while 2 (l_max + 1) < 80."""
    from oracle import angular
    l_max = 6
    D = _three_pols(2, l_max, seed=8)
    n = (l_max + 1) ** 2
    lms = [angular.idx_to_lm(i) for i in range(n)]
    qs = (1, -1, 0)                                           # x, y, z
    exact = []
    for e in range(2):
        sig = sum(np.sum(np.abs(d[e]) ** 2) for d in D) / 3.0
        amp = {}
        for qi, q in enumerate(qs):
            for i, (l, m) in enumerate(lms):
                for lam in (l - 1, l + 1):
                    if lam < 0:
                        continue
                    for mlam in range(-lam, lam + 1):
                        g = angular.gaunt_real(l, m, 1, q, lam, mlam)
                        if g != 0.0:
                            amp[(lam, mlam)] = amp.get((lam, mlam), 0.0) + D[qi][e, i] * g
        N1 = 4.0 * np.pi / 3.0 * sum(abs(a) ** 2 for a in amp.values())
        exact.append(N1 / sig - 1.0)
    assert np.allclose(OBS.beta(*D), exact, rtol=1e-12, atol=1e-13)


def test_scan_observables_on_solver_shaped_results():
    """scan_observables reads .E and .D (six slots of N_psi dipoles) of the
    solver's per-energy results, sorts them by energy and returns every
    observable keyed by gauge and polarisation."""
    from types import SimpleNamespace
    rng = np.random.default_rng(9)
    n_mu, Es = 9, [0.9, 0.5, 0.7, 0.6]
    res = [SimpleNamespace(E=E, D=[rng.standard_normal(n_mu) + 1j * rng.standard_normal(n_mu) for _ in range(6)])
           for E in Es]
    obs = OBS.scan_observables(res, e_homo=-0.6)
    order = np.argsort(Es)
    k = np.sqrt(2.0 * np.array(Es)[order])
    assert np.allclose(obs["k"], k)
    for s, (gauge, pol) in enumerate(OBS.SLOTS):
        D = np.stack([res[i].D[s] for i in order])
        assert np.allclose(obs[f"sigma_{gauge}_{pol}"], OBS.cross_section(k, D, obs["omega"], gauge))
        assert np.allclose(obs[f"tau_{gauge}_{pol}"], OBS.time_delay(k, D))
    for p, pol in enumerate("xyz"):
        DL = np.stack([res[i].D[p] for i in order])
        DV = np.stack([res[i].D[3 + p] for i in order])
        assert np.allclose(obs[f"dphi_rms_{pol}"], OBS.dphi_rms(DL, DV))
    for g, gauge in enumerate(("length", "velocity")):
        b = obs[f"beta_{gauge}"]
        assert b.shape == (len(Es),) and np.all((b >= -1 - 1e-12) & (b <= 2 + 1e-12))


def test_against_the_reference_code():
    """tests/golden/observables_vectors.json holds seeded dipoles and what the
    reference's own postprocessing/cross_section_delay.py computed from them
    (tests/golden/make_observables_golden.py): sigma, tau in both sign
    conventions, q, dphi_rms and beta."""
    import json
    import os
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "observables_vectors.json")))
    k, om = np.array(g["k"]), np.array(g["omega"])
    D = [np.array(re) + 1j * np.array(im) for re, im in zip(g["D_re"], g["D_im"])]
    for s, (gauge, pol) in enumerate(OBS.SLOTS):
        assert np.allclose(OBS.cross_section(k, D[s], om, gauge), g[f"sigma_{gauge}_{pol}"], rtol=1e-14, atol=0)
        assert np.allclose(OBS.time_delay(k, D[s]), g[f"tau_{gauge}_{pol}"], rtol=1e-13, atol=1e-15)
        assert np.allclose(OBS.time_delay(k, D[s], with_minus=True), g[f"tau_minus_{gauge}_{pol}"],
                           rtol=1e-13, atol=1e-15)
    for p, pol in enumerate("xyz"):
        assert np.allclose(OBS.q_sigma(D[p], D[3 + p], om), g[f"q_{pol}"], rtol=1e-14, atol=0)
        assert np.allclose(OBS.dphi_rms(D[p], D[3 + p]), g[f"dphi_rms_{pol}"], rtol=1e-14, atol=0)
    for i, gauge in enumerate(("length", "velocity")):
        assert np.allclose(OBS.beta(D[3 * i], D[3 * i + 1], D[3 * i + 2]), g[f"beta_{gauge}"], rtol=1e-12, atol=1e-14)

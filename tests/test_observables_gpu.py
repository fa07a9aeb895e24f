"""Scan observables (cross sections, Wigner delays, gauge ratio) from the CUDA
solver's dipoles against the same observables from the oracle's dipoles."""
import numpy as np
import pytest

from oracle import solver as O
from scatt_b200 import observables as OBS
from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu


def test_scan_observables_match_oracle():
    inp = synth.h2_like(Nr=801, dr=0.05, l_cont=2)
    ks = np.linspace(0.6, 1.4, 7)
    Es = 0.5 * ks ** 2
    sol = S.ScanSolver(inp)
    got = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1))
    e_homo = -0.6
    obs = OBS.scan_observables(got, e_homo)
    st = O.make_setup(inp)
    ref = [O.solve_energy(st, E) for E in Es]
    om = Es - e_homo
    for s, (gauge, pol) in enumerate(OBS.SLOTS):
        Dref = np.stack([r.slices[s]["D"] for r in ref])
        sig = OBS.cross_section(ks, Dref, om, gauge)
        tau = OBS.time_delay(ks, Dref)
        assert np.max(np.abs(obs[f"sigma_{gauge}_{pol}"] - sig)) <= 1e-9 * max(np.max(np.abs(sig)), 1e-300)
        # the delay divides by sum |D|^2 and differences neighbouring energies
        assert np.max(np.abs(obs[f"tau_{gauge}_{pol}"] - tau)) <= 1e-8 * max(np.max(np.abs(tau)), 1.0)

"""Tournament pivoting (oracle/pivoting.py), the planned device panel scheme,
against partial pivoting: the inverse on its own, and the whole solve with
every dense inverse of the oracle replaced by it.

In the solve the change is held to the spread between the oracle's two
LAPACK builds (eigen: partial-pivot LU; mkl: dgetri and dsytrf/dsytri),
the floor the GPU parity tolerances already sit on.  The two differences
point the same way (correlation above 0.9): any change of rounding is
amplified along the same ill-conditioned directions of the problem, so the
pivot order does not move the floor.
"""
import numpy as np
import pytest

from oracle import pivoting
from oracle import solver as O
from scatt_b200 import synth


@pytest.mark.parametrize("n", [5, 17, 50, 163])
def test_tournament_inverse(n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 0.1 * np.eye(n)
    X = pivoting.gj_inverse_tournament(A)
    assert np.max(np.abs(A @ X - np.eye(n))) < 1e-11
    ref = np.linalg.inv(A)
    assert np.max(np.abs(X - ref)) <= 1e-11 * np.max(np.abs(ref))


def _solve(inp, E, mode, monkeypatch):
    with monkeypatch.context() as m:
        m.setattr(O, "BUILD", "mkl" if mode == "mkl" else "eigen")
        if mode == "tournament":
            m.setattr(O, "inverse_general", pivoting.gj_inverse_tournament)
        return O.solve_energy(O.make_setup(inp), E)


@pytest.mark.parametrize("E", [0.3, 1.5])
def test_solve_with_tournament_pivoting_stays_at_the_build_floor(monkeypatch, E):
    inp = synth.h2_like(Nr=401, dr=0.1, l_cont=4)
    base, mkl, tour = (_solve(inp, E, m, monkeypatch) for m in ("eigen", "mkl", "tournament"))
    dK_t = tour.K_kme - base.K_kme
    dK_m = mkl.K_kme - base.K_kme
    scale = np.max(np.abs(base.K_kme))
    assert 0.0 < np.max(np.abs(dK_t)) <= 3.0 * max(np.max(np.abs(dK_m)), 1e-15 * scale)
    corr = np.sum(dK_t * dK_m) / np.sqrt(np.sum(dK_t ** 2) * np.sum(dK_m ** 2))
    assert corr > 0.9                     # 0.977 at E = 0.3, 0.99997 at E = 0.8
    for s in range(6):
        d_t = np.max(np.abs(tour.slices[s]["D"] - base.slices[s]["D"]))
        d_m = np.max(np.abs(mkl.slices[s]["D"] - base.slices[s]["D"]))
        ref = np.max(np.abs(base.slices[s]["D"]))
        assert d_t <= max(3.0 * d_m, 1e-12 * ref)

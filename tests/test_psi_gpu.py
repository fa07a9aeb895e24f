"""psi(n) reconstruction (scatt_psi_sweep: the reference's BackPropagator::run
+ get_psi, src/scatt/BackPropagator.cpp:199-802) against the oracle's
back-propagation, through the C ABI.

The oracle keeps psi(n) for n <= n_transition - 1 and over the 300-point
asymptotic tail (BackPropagator.cpp:502-531, oracle/solver.py solve_energy);
the device sweep is compared at those points.  Tolerance: max(1e-10,
10 x floor), the floor being how far the oracle's own psi moves between the
reference's two LAPACK builds or the floor of K, A and B (psi descends from
the boundary value psi_N = J + Y K), whichever is larger.  Segment sizes,
sub-ranges and host buffers change no arithmetic, so they agree to 1e-12.
"""
import numpy as np
import pytest

from oracle import solver as O
from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def h2():
    inp = synth.h2_like(Nr=801, dr=0.05, l_cont=2)
    sol = S.ScanSolver(inp, device=0)
    yield inp, sol
    sol.close()


def test_psi_matches_oracle_back_sweep(h2):
    inp, sol = h2
    Es = [0.125, 0.5, 1.2]
    res, psi = sol.psi_sweep(Es, segment=64, opts=S.default_opts(allow_closed_channels=1))
    assert psi.shape == (3, inp.Nr, sol.Np, sol.Np)
    st = O.make_setup(inp)
    Np = st.n_mu
    fails = []
    for i, E in enumerate(Es):
        O.BUILD = "eigen"
        r = O.solve_energy(st, E, keep_psi=True)
        O.BUILD = "mkl"
        r2 = O.solve_energy(st, E, keep_psi=True)
        O.BUILD = "eigen"
        ns = sorted(r.psi_keep)
        assert ns[0] == 0 and ns[-1] == inp.Nr - 1
        ref = np.stack([r.psi_keep[n] for n in ns])
        alt = np.stack([r2.psi_keep[n] for n in ns])
        got = np.stack([psi[i, n, :Np, :Np] for n in ns])
        coupled = max(rel(r2.K_kme, r.K_kme), rel(r2.aa["A"], r.aa["A"]), rel(r2.aa["B"], r.aa["B"]))
        floor = max(rel(alt, ref), coupled)
        tol = max(1e-10, 10.0 * floor)
        err = rel(got, ref)
        if not err <= tol:
            fails.append(f"E={E} psi err {err:.3e} floor {floor:.3e}")
        if not rel(res[i].K_kme, r.K_kme) <= tol:
            fails.append(f"E={E} K err {rel(res[i].K_kme, r.K_kme):.3e}")
        assert res[i].status == 0
    assert not fails, "\n".join(fails)


def test_psi_segments_ranges_and_results_agree(h2):
    """Segments of 8 and 64 steps, a sub-range, and the batch solver's own
    results (fit accumulated forward) give the same numbers."""
    inp, sol = h2
    Es = [0.3, 0.9]
    o = S.default_opts(allow_closed_channels=1)
    res, full = sol.psi_sweep(Es, segment=64, opts=o)
    _, p8 = sol.psi_sweep(Es, segment=8, opts=o)
    _, part = sol.psi_sweep(Es, n_lo=137, n_hi=611, segment=32, opts=o)
    assert rel(p8, full) <= 1e-12
    assert part.shape[1] == 611 - 137
    assert rel(part, full[:, 137:611]) <= 1e-12
    assert np.max(np.abs(full)) > 0 and np.all(np.isfinite(full))
    ref = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1, keep_window=0))
    for g, r in zip(res, ref):
        assert rel(g.K_kme, r.K_kme) <= 1e-12
        assert rel(g.A, r.A) <= 1e-12 and rel(g.B, r.B) <= 1e-12
        assert rel(g.D, r.D) <= 1e-12


def test_psi_into_page_locked_host_memory(h2):
    """The copies from page-locked memory overlap the sweep; the numbers are
    those of a pageable buffer."""
    torch = pytest.importorskip("torch")
    inp, sol = h2
    keep = []

    def pinned(shape, dtype=np.float64):
        t = torch.zeros(shape, dtype=torch.float64, pin_memory=True)
        keep.append(t)
        return t.numpy()

    o = S.default_opts(allow_closed_channels=1)
    _, a = sol.psi_sweep([0.7], n_lo=300, segment=16, opts=o)
    _, b = sol.psi_sweep([0.7], n_lo=300, segment=16, opts=o, alloc=pinned)
    assert rel(b, a) <= 1e-12


def test_psi_mixed_l_cont_blocks():
    """Energies with different continuum cutoffs in one sweep: each fills
    its own Np x Np block, zero elsewhere, and equals the sweep of that
    energy alone.  A lone energy of the smaller cutoff runs on smaller
    batch shapes, whose GEMM tiles may round differently, and the recurrence
    amplifies rounding to about 1e-8 of psi on such cases: hence 1e-8."""
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=11, lmax_orb=8, n_orb=2)
    sol = S.ScanSolver(inp, device=0)
    o = S.default_opts(allow_closed_channels=1)
    Es, lcs = [0.4, 0.9], [10, 11]
    _, mix = sol.psi_sweep(Es, l_cont=lcs, segment=40, opts=o)
    for i, (E, lc) in enumerate(zip(Es, lcs)):
        n = (lc + 1) ** 2
        _, one = sol.psi_sweep([E], l_cont=[lc], segment=40, opts=o)
        assert rel(mix[i, :, :n, :n], one[0, :, :n, :n]) <= 1e-8
        assert np.all(mix[i, :, n:, :] == 0.0) and np.all(mix[i, :, :, n:] == 0.0)
    sol.close()


def test_psi_sweep_rejects_bad_ranges(h2):
    _, sol = h2
    from scatt_b200._lib import ScattError
    for kw in (dict(n_lo=5, n_hi=5), dict(n_lo=-1), dict(n_hi=inp_nr_plus_one(sol)), dict(segment=12)):
        with pytest.raises(ScattError):
            sol.psi_sweep([0.5], **kw)


def inp_nr_plus_one(sol):
    return sol.inp.Nr + 1

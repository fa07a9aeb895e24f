"""Streaming scan (scatt_scan_*) through the C ABI, against the batch solve.

The scan runs the same kernels on the same per-energy data as
scatt_solve_batch, only with energies entering and leaving in phase-staggered
groups, so every energy's results must equal the batch solve's: the tests
hold them to 1e-13 relative (in practice they agree bit for bit).  Chunk
replay from CUDA graphs (opts.use_graphs) is held to the same bar.
"""
import numpy as np
import pytest

from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu

FIELDS = ("K_kme", "A", "B", "K_aa", "b_overlap", "D", "D_raw", "d_raw", "d_corr", "partial_sigma")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def drain(scan):
    got, order = {}, []
    while True:
        r = scan.step()
        if not r:
            return got, order
        order.append([i for i, _ in r])
        got.update(dict(r))


def same(g, r, tag):
    for f in FIELDS:
        assert rel(getattr(g, f), getattr(r, f)) < 1e-13, f"{tag} {f}"
    for k in ("shifts_A", "shifts_S", "n_closed_l", "n_fit_start", "n_fit_end"):
        assert g.diag[k] == r.diag[k], f"{tag} {k}"
    assert g.status == r.status == 0


def test_scan_equals_batch_staggered():
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=3)
    sol = S.ScanSolver(inp)
    opts = S.default_opts(allow_closed_channels=1)
    Es = [0.2, 0.45, 0.8, 1.1, 1.5, 1.9, 0.33]
    ref = sol.solve(Es, opts=opts)
    scan = sol.scan(slots=3, groups=3, opts=opts)
    assert (scan.slots, scan.groups) == (3, 3)
    assert scan.submit(Es) == list(range(len(Es)))
    got, order = drain(scan)
    assert sorted(got) == list(range(len(Es)))
    # one slot per group: energies leave one at a time, in the order they entered
    assert [i for o in order for i in o] == list(range(len(Es)))
    for i, E in enumerate(Es):
        assert got[i].E == E
        same(got[i], ref[i], f"E={E}")
    assert scan.pending() == (0, 0)
    scan.close()


def test_scan_groups_of_two_and_refill_after_drain():
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=3)
    sol = S.ScanSolver(inp)
    opts = S.default_opts(allow_closed_channels=1)
    Es1, Es2 = [0.3, 0.9, 1.4, 0.6, 1.7], [0.75, 1.25]
    ref = sol.solve(Es1 + Es2, opts=opts)
    scan = sol.scan(slots=4, groups=2, opts=opts)
    scan.submit(Es1)
    got, _ = drain(scan)
    assert scan.pending() == (0, 0)
    scan.submit(Es2)                           # idle groups start again at once
    got2, _ = drain(scan)
    got.update(got2)
    assert sorted(got) == list(range(7))
    for i, r in enumerate(ref):
        same(got[i], r, f"E={r.E}")


def test_scan_mixed_l_cont():
    """Energies with continuum cutoffs 10 and 11 share the scan's slots."""
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=11, lmax_orb=8, n_orb=2)
    sol = S.ScanSolver(inp)
    opts = S.default_opts(allow_closed_channels=1)
    Es, lcs = [0.4, 0.9, 0.6, 1.3], [10, 11, 11, 10]
    ref = sol.solve(Es, l_cont=lcs, opts=opts)
    scan = sol.scan(slots=2, groups=2, opts=opts)
    scan.submit(Es, l_cont=lcs)
    got, _ = drain(scan)
    for i in range(len(Es)):
        assert got[i].K_kme.shape == ((lcs[i] + 1) ** 2,) * 2
        same(got[i], ref[i], f"l={lcs[i]} E={Es[i]}")


def test_scan_rejects_bad_requests():
    # l_cont 11 uploaded: the exchange cutoff min(l, 10) = 10 is shared, so a
    # scan may be opened at l_cont_max 10 and 11 but not below 10
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=11, lmax_orb=8, n_orb=2)
    sol = S.ScanSolver(inp)
    with pytest.raises(Exception):
        sol.scan(slots=2, groups=65)
    with pytest.raises(Exception):
        sol.scan(slots=2, groups=1, l_cont_max=9)
    scan = sol.scan(slots=2, groups=1, l_cont_max=10)
    with pytest.raises(Exception):
        scan.submit([0.5], l_cont=[11])         # above the scan's l_cont_max
    with pytest.raises(Exception):
        scan.submit([-0.1])
    assert scan.step() == []                    # nothing queued
    scan.close()


def test_graph_replay_equals_direct_launches():
    """opts.use_graphs replays each chunk from a captured CUDA graph: the
    same kernels with the same arguments, so the same results."""
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)
    sol = S.ScanSolver(inp)
    Es = [0.3, 0.7, 1.1, 1.6]
    ref = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1))
    got = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1, use_graphs=1))
    for r, g in zip(ref, got):
        same(g, r, f"batch E={r.E}")
    scan = sol.scan(slots=2, groups=2, opts=S.default_opts(allow_closed_channels=1, use_graphs=1, timing=1))
    scan.submit(Es)
    res, _ = drain(scan)
    for i, r in enumerate(ref):
        same(res[i], r, f"scan E={r.E}")


@pytest.mark.parametrize("builder,kw,Es", [
    ("h2o_like", dict(Nr=301, dr=0.05, l_cont=4, lmax_orb=8, n_orb=3), [0.3, 0.7, 1.1]),
    ("h2_like", dict(Nr=401, dr=0.05, l_cont=8), [0.5 * 0.08 ** 2, 0.6]),     # l = 8 closed at k = 0.08
])
def test_forward_fit_accumulation_equals_window_sweep(builder, kw, Es):
    """keep_window = 0 accumulates the amplitude fit forward ([A; B] =
    G_A(N-1)^T Z_N) instead of sweeping psi back over the stored window:
    the same A, B, K and dipoles up to the order of summation; the fit
    residual (it needs psi at every window point) is then NaN."""
    inp = getattr(synth, builder)(**kw)
    sol = S.ScanSolver(inp)
    ref = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1))
    got = sol.solve(Es, opts=S.default_opts(allow_closed_channels=1, keep_window=0))
    for r, g in zip(ref, got):
        assert np.array_equal(g.K_kme, r.K_kme)          # the same R-ratios and K extraction
        for f in ("A", "B", "K_aa", "b_overlap", "D", "D_raw", "d_raw", "partial_sigma"):
            assert rel(getattr(g, f), getattr(r, f)) < 1e-11, (builder, r.E, f)
        assert g.diag["n_closed_l"] == r.diag["n_closed_l"]
        assert np.isnan(g.diag["fit_residual_max"]) and np.isnan(g.diag["fit_residual_rel"])
    # and through a staggered scan
    scan = sol.scan(slots=2, groups=2, opts=S.default_opts(allow_closed_channels=1, keep_window=0))
    scan.submit(Es)
    res, _ = drain(scan)
    for i, r in enumerate(ref):
        assert rel(res[i].A, r.A) < 1e-11 and rel(res[i].D, r.D) < 1e-11

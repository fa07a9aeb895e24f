"""A scan read from a preprocessing file gives the results of the same inputs
handed over directly, and its results survive the dipole scan files."""
import numpy as np
import pytest

from scatt_b200 import h5io
from scatt_b200 import solver as S
from scatt_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("split", [False, True])
def test_preproc_scan_equals_direct_inputs(tmp_path, split):
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=4, lmax_orb=8, n_orb=3)
    path = h5io.write_preproc(tmp_path / "m", inp, split=split)
    opts = S.default_opts(allow_closed_channels=1)
    ks = np.array([0.5, 0.9, 1.3])
    ref = S.ScanSolver(inp).solve(0.5 * ks ** 2, opts=opts)
    sol = S.ScanSolver.from_preproc(path, l_cont_max=4)
    assert sol.E_init == inp.orb_energies[inp.n_occ - 1]
    got = sol.solve(0.5 * ks ** 2, opts=opts)
    for r, g in zip(ref, got):
        for f in ("K_kme", "A", "B", "b_overlap", "D_raw", "d_raw"):
            np.testing.assert_array_equal(getattr(g, f), getattr(r, f), err_msg=f)
        # each solver builds its own d_correction table, whose sums over the
        # channels run in shared-memory atomic order: D, d_corr and sigma to rounding
        for f in ("D", "d_corr", "partial_sigma"):
            a, b = getattr(g, f), getattr(r, f)
            assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b)), f
    meta = h5io.scan_meta(inp, dk=0.1, ik_min=1, ik_max=20)
    h5io.write_dipole_scan(tmp_path / "scan", meta, [(int(round(k / 0.1)), g) for k, g in zip(ks, got)])
    rd = h5io.DipoleReader(tmp_path / "scan")
    assert rd.available_ik() == [5, 9, 13]
    back = rd.read_energy(9)
    np.testing.assert_array_equal(back["A"], got[1].A)
    np.testing.assert_array_equal(back["slices"][5]["D"], got[1].D[5])

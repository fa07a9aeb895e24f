"""The library's angular grid of the single-centre expansion
(scatt_sce_grid, host-only) equals the oracle's: numpy's Gauss-Legendre
nodes and weights in cos(theta), ascending, and phi_j = 2 pi j / n_phi
(preprocessing/src/angular/Grid.hpp, GaussLegendre.hpp)."""
import numpy as np
import pytest

from oracle import sce as SC
from scatt_b200 import _lib


@pytest.mark.parametrize("Lmax", [0, 1, 4, 10, 40, 120])
def test_grid_matches_numpy_gauss_legendre(Lmax):
    x, w, phi = _lib.sce_grid(Lmax)
    xr, wr, _, pr = SC.grid(Lmax)
    assert np.all(np.diff(x) > 0)
    assert np.max(np.abs(x - xr)) <= 1e-15
    assert np.max(np.abs(w - wr)) <= 1e-14
    assert np.array_equal(phi, pr)
    assert abs(w.sum() - 2.0) <= 1e-13

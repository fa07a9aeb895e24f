"""The device single-centre expansion (scatt_sce_project: the projection of
preprocessing/src/sce/SCE.hpp:122-266 as two DMMA GEMM stages) against the
oracle's restatement (oracle/sce.py, held to closed forms and exact
recovery in tests/test_oracle_sce.py).  Same quadrature, different
summation order: 1e-12 of the largest coefficient.  Chunk sizes of one,
three and all radial points; grids up to Lmax = 130, where the Legendre
step's GEMM takes the 128-row tiles."""
import numpy as np
import pytest

from oracle import sce as SC
from scatt_b200 import _lib

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("Lmax,Nr,chunk", [(0, 3, 0), (4, 7, 3), (12, 11, 1), (40, 9, 0), (130, 4, 3)])
def test_sce_projection_matches_oracle(Lmax, Nr, chunk):
    rng = np.random.default_rng(Lmax * 100 + Nr)
    X = rng.standard_normal((Nr, Lmax + 1, 2 * (Lmax + 1)))
    got = _lib.sce_project(X, Lmax, chunk)
    ref = SC.project(X, Lmax)
    assert got.shape == ref.shape
    assert rel(got, ref) <= 1e-12


def test_sce_recovers_band_limited_coefficients():
    rng = np.random.default_rng(9)
    Lmax, Lf = 10, 8
    coef = rng.standard_normal(((Lf + 1) ** 2, 5))
    got = _lib.sce_project(SC.synthesize(coef, Lmax), Lmax, chunk=2)
    want = np.zeros(((Lmax + 1) ** 2, 5))
    want[:coef.shape[0]] = coef
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(coef))

"""The device basis-to-expansion path (scatt_sce_basis: the AO values of
preprocessing/src/basis/MoldenBasis.hpp, the orbitals and the density, each
and the local exchange of potential/LocalExchange.hpp, each projected as
preprocessing/src/sce/SCE.hpp does) against the oracle
(oracle/basis.py with oracle/sce.py, pinned in tests/test_oracle_basis.py
and tests/test_oracle_sce.py).  Same arithmetic up to summation order and
the angles (the device forms cos / sin of theta and phi algebraically, the
oracle through arccos / arctan2): 1e-12 of each function's largest
coefficient."""
import numpy as np
import pytest

from oracle import basis as B
from scatt_b200 import _lib

pytestmark = pytest.mark.gpu


def _molecule(seed=11):
    rng = np.random.default_rng(seed)
    centres = [np.zeros(3), np.array([0.0, 1.43, 1.1]), np.array([0.0, -1.43, 1.1])]
    shells = []
    for a, c in enumerate(centres):
        for l in range(3 if a == 0 else 2):
            n = 1 + (l + a) % 3
            shells.append((c, l, np.sort(rng.uniform(0.15, 6.0, n))[::-1], rng.uniform(0.2, 1.0, n)))
    nbf = sum(1 if s[1] == 0 else 2 * s[1] + 1 for s in shells)
    C = rng.standard_normal((4, nbf))
    occ = np.array([2.0, 2.0, 2.0, 0.0])
    return shells, C, occ


@pytest.mark.parametrize("Lmax,Nr,chunk,r0,vx", [(6, 9, 0, 0.0, 0), (10, 13, 4, 0.02, 1), (16, 5, 1, 0.0, 2)])
def test_basis_expansions_match_oracle(Lmax, Nr, chunk, r0, vx):
    """Orbitals, density and (Slater or Kohn-Sham) local exchange."""
    shells, C, occ = _molecule()
    dr = 0.3
    origin = np.array([0.0, 0.0, 0.35])
    got = _lib.sce_basis(shells, C, occ, Lmax, Nr, r0, dr, origin, chunk, vx_form=vx)
    r = r0 + np.arange(Nr) * dr
    ref = B.sce_of_basis(shells, C, occ, Lmax, r, origin, vx_form=vx)
    assert len(got) == len(ref) == (3 if vx else 2)
    for i in range(C.shape[0]):
        scale = np.max(np.abs(ref[0][i]))
        assert np.max(np.abs(got[0][i] - ref[0][i])) <= 1e-12 * scale, i
    for g, f in zip(got[1:], ref[1:]):
        assert np.max(np.abs(g - f)) <= 1e-12 * np.max(np.abs(f))

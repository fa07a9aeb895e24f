"""The oracle solved on a symmetry block of continuum channels equals that
block of the full solve.

On a linear molecule on the z axis the static-exchange potential couples
(l, m) only to (l', m) with l + l' even, so the channels fall into blocks
(sigma_g: m = 0, l even; pi: m = +-1, ...).  make_setup(channels=...)
keeps one block: V, the exchange rows and the per-channel tables are those
of the kept channels.  The reference always solves every channel; the
subset is the groundwork for a block-diagonal device solve, and this test
pins what it must reproduce.  The stability shift of
SchurInverter.cpp:53-59 is decided on the whole matrix, that is on the
lowest eigenvalue over every block; decided on the block alone
(whole_matrix_shift=False) it can differ, and the sigma_u case shows how.
"""
import numpy as np
import pytest

from oracle import solver as O
from scatt_b200 import synth

E = 0.6


@pytest.fixture(scope="module")
def full():
    inp = synth.h2_like(Nr=201, dr=0.05, l_cont=4)
    return inp, O.solve_energy(O.make_setup(inp), E)


def block(inp, channels, whole=True):
    return O.solve_energy(O.make_setup(inp, channels=channels, whole_matrix_shift=whole), E)


@pytest.mark.parametrize("channels", [[0, 6, 20], [2, 12], [1, 5, 11, 19], [3, 7, 13, 21]],
                         ids=["sigma_g", "sigma_u", "pi_minus", "pi_plus"])
def test_block_equals_the_full_solve(full, channels):
    inp, rf = full
    rs = block(inp, channels)
    assert rs.shifts == rf.shifts
    S = np.array(channels)
    other = np.setdiff1d(np.arange(rf.K_kme.shape[0]), S)
    assert np.max(np.abs(rf.K_kme[np.ix_(S, other)])) == 0.0      # the block is closed
    scale = np.max(np.abs(rs.K_kme))
    assert np.max(np.abs(rf.K_kme[np.ix_(S, S)] - rs.K_kme)) <= 1e-11 * scale
    for q in range(6):
        Df, Ds = rf.slices[q]["D"], rs.slices[q]["D"]
        assert Ds.shape == (S.size,)
        tol = 1e-8 * max(np.max(np.abs(Ds)), 1e-300)
        assert np.max(np.abs(Df[S] - Ds)) <= tol, q


def test_shift_decided_on_the_block_alone_differs(full):
    """sigma_u (m = 0, l odd): the full solve shifts A once (at n = 1, by
    another block's lowest eigenvalue); the block decided alone does not.
    n = 1 lies in the analytic start of the forward recurrence, so K still
    agrees, but the back-propagation runs through S^-1(1), so psi near the
    origin and the dipoles that see it differ."""
    inp, rf = full
    S = [2, 12]
    rs = block(inp, S, whole=False)
    assert rf.shifts == {"A": 1, "S": 0} and rs.shifts == {"A": 0, "S": 0}
    assert np.max(np.abs(rf.K_kme[np.ix_(S, S)] - rs.K_kme)) <= 1e-11 * np.max(np.abs(rs.K_kme))
    rel = [np.max(np.abs(rf.slices[q]["D"][S] - rs.slices[q]["D"])) / np.max(np.abs(rs.slices[q]["D"]))
           for q in range(6) if np.max(np.abs(rs.slices[q]["D"])) > 0]
    assert rel and 1e-8 < max(rel) < 1e-3


def test_bad_channel_lists_raise():
    inp = synth.h2_like(Nr=41, dr=0.05, l_cont=2)
    for bad in ([], [-1], [9]):
        with pytest.raises(ValueError):
            O.make_setup(inp, channels=bad)

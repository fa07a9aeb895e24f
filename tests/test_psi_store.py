"""The psi store on disk (scatt_psi_store_*, the layout the reference's
BackPropagator writes and its continuum-continuum dipole driver reads:
src/scatt/BackPropagator.cpp:27-101, :255-283; PotentialStorage.cpp:31-35,
:556-631, :1542-1566), checked byte by byte with an independent parser
here, plus the round trip through the library's reader.  Host-only."""
import os
import struct

import numpy as np
import pytest

from scatt_b200 import psi_store as PS
from scatt_b200._lib import ScattError


def _meta(**kw):
    base = dict(energy=0.72, dr=0.005, n_grid=12001, n_psi=5, n_f=7, l_cont=1, l_exch=1, n_occ=2,
                n_transition=600, keep_lo=0, keep_hi=10, chunk_size=4)
    base.update(kw)
    return PS.meta(**base)


def test_store_bytes_and_round_trip(tmp_path):
    rng = np.random.default_rng(7)
    L = 8                                   # psi_sweep's ld (Np_max) above the store's N_psi = 5
    psi = np.zeros((11, L, L))
    psi[:, :5, :5] = rng.standard_normal((11, 5, 5))
    asym = rng.standard_normal((3, 5, 5))
    m = _meta(asym_offset=9000)
    d = tmp_path / PS.dirname(m)
    assert d.name == "psi_Nr12001_Npsi5_E0.720000_lc1_keep0-10"
    PS.write(d, m, psi, asym)
    assert sorted(os.listdir(d)) == ["__SUCCESS__", "manifest.txt", "metadata.bin", "pot_chunk_0.bin",
                                     "pot_chunk_1.bin", "pot_chunk_2.bin", "psi_asym.bin"]
    assert (d / "manifest.txt").read_text() == ("kind=psi energy=0.720000 Nr=12001 dr=0.005000 Npsi=5 Nf=7 "
                                                "l_cont=1 l_exch=1 n_occ=2 n_trans=600 keep=0..10")
    assert struct.unpack("<Qiii", (d / "metadata.bin").read_bytes()) == (11, 5, 4, 3)
    got = []
    for c, n in ((0, 4), (1, 4), (2, 3)):
        raw = (d / f"pot_chunk_{c}.bin").read_bytes()
        assert struct.unpack_from("<i", raw)[0] == n and len(raw) == 4 + n * 25 * 8
        mats = np.frombuffer(raw, dtype="<f8", offset=4).reshape(n, 5, 5)
        got.append(np.swapaxes(mats, 1, 2))             # column-major on disk
    np.testing.assert_array_equal(np.concatenate(got), psi[:, :5, :5])
    raw = (d / "psi_asym.bin").read_bytes()
    assert raw[:8] == b"PSI_ASYM" and struct.unpack_from("<iiiiq", raw, 8) == (1, 3, 9000, 5, 0)
    np.testing.assert_array_equal(np.swapaxes(np.frombuffer(raw, "<f8", offset=32).reshape(3, 5, 5), 1, 2), asym)
    with PS.Store(d) as s:
        assert (s.points, s.n_psi, s.chunk_size, s.chunks, s.n_asym, s.asym_offset) == (11, 5, 4, 3, 3, 9000)
        assert s.manifest.startswith("kind=psi energy=0.720000")
        np.testing.assert_array_equal(s.read(), psi[:, :5, :5])
        np.testing.assert_array_equal(s.read(3, 6), psi[3:9, :5, :5])   # across chunk boundaries
        np.testing.assert_array_equal(s.asym(), asym)


def test_store_without_success_marker_is_refused(tmp_path):
    m = _meta(keep_hi=2)
    PS.write(tmp_path / "s", m, np.ones((3, 5, 5)))
    assert not (tmp_path / "s" / "psi_asym.bin").exists()
    os.remove(tmp_path / "s" / "__SUCCESS__")
    with pytest.raises(ScattError, match="__SUCCESS__") as e:
        PS.Store(tmp_path / "s")
    assert e.value.code == 11


def test_bad_arguments(tmp_path):
    with pytest.raises(ScattError):                     # matrices smaller than N_psi
        PS.write(tmp_path / "x", _meta(keep_hi=2), np.ones((3, 4, 4)))
    with pytest.raises(ValueError):
        PS.write(tmp_path / "y", _meta(keep_hi=4), np.ones((3, 5, 5)))
    with PS.Store(PS.write(tmp_path / "z", _meta(keep_hi=1), np.ones((2, 5, 5)))) as s:
        with pytest.raises(ScattError):
            s.read(1, 5)

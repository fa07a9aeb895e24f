"""HDF5 subset, dipole scan output and preprocessing input (CPU only).

The library's writer is checked twice: by its own reader (round trips) and by
`Walk`, an independent parser in this file that follows the HDF5 file-format
specification for the structures the writer claims to emit (superblock 0,
version-1 object headers, symbol-table groups with their local heap, B-tree
and symbol-table nodes, contiguous and deflate-chunked layouts, version-1
attribute messages).  The dipole layout is the reference's DipoleWriter
(src/scatt/DipoleIO.cpp:141-336); the preprocessing schema its HDF5Reader
(src/io/HDF5Reader.hpp:446-570).
"""
import os
import struct
import types
import zlib

import numpy as np
import pytest

from scatt_b200 import _lib, h5io, synth


# ---------------------------------------------------------------- independent parser
class Walk:
    SIG = b"\x89HDF\r\n\x1a\n"

    def __init__(self, path):
        self.b = open(path, "rb").read()
        assert self.b[:8] == self.SIG
        assert self.b[8] == 0                     # superblock version 0
        assert self.b[13] == 8 and self.b[14] == 8
        self.leaf_k, self.node_k = struct.unpack_from("<HH", self.b, 16)
        eof = struct.unpack_from("<Q", self.b, 40)[0]
        assert eof == len(self.b)
        self.root = struct.unpack_from("<Q", self.b, 64)[0]

    def u(self, fmt, at):
        return struct.unpack_from("<" + fmt, self.b, at)

    def header(self, at):
        ver, _, n, _, size = self.u("BBHII", at)
        assert ver == 1
        msgs, p = [], at + 16
        for _ in range(n):
            t, sz, _ = self.u("HHI", p)
            assert sz % 8 == 0
            msgs.append((t, self.b[p + 8:p + 8 + sz]))
            p += 8 + sz
        assert p == at + 16 + size
        return msgs

    def links(self, at):
        st = [m for t, m in self.header(at) if t == 0x11]
        assert len(st) == 1
        bt, heap = struct.unpack_from("<QQ", st[0])
        assert self.b[heap:heap + 4] == b"HEAP"
        hsize, free, data = self.u("QQQ", heap + 8)
        assert free == 1
        names = self.b[data:data + hsize]
        assert self.b[bt:bt + 4] == b"TREE" and self.b[bt + 4] == 0 and self.b[bt + 5] == 0
        used = self.u("H", bt + 6)[0]
        assert used <= 2 * self.node_k
        out, prev_last = [], b""
        for i in range(used):
            key_lo = self.u("Q", bt + 24 + 16 * i)[0]
            child = self.u("Q", bt + 32 + 16 * i)[0]
            key_hi = self.u("Q", bt + 40 + 16 * i)[0]
            assert names[key_lo:].split(b"\0")[0] == prev_last
            assert self.b[child:child + 4] == b"SNOD"
            n = self.u("H", child + 6)[0]
            assert 0 < n <= 2 * self.leaf_k
            ents = []
            for k in range(n):
                off, hdr = self.u("QQ", child + 8 + 40 * k)
                ents.append((names[off:].split(b"\0")[0], hdr))
            assert [e[0] for e in ents] == sorted(e[0] for e in ents)
            assert names[key_hi:].split(b"\0")[0] == ents[-1][0]
            prev_last = ents[-1][0]
            out += ents
        return {k.decode(): v for k, v in out}

    def resolve(self, path):
        at = self.root
        for part in [p for p in path.split("/") if p]:
            at = self.links(at)[part]
        return at

    @staticmethod
    def dtype(m):
        cls, size = m[0] & 0x0F, struct.unpack_from("<I", m, 4)[0]
        if cls == 1:
            assert m[1:4] == b"\x20\x3f\x00" and size == 8
            assert struct.unpack_from("<HHBBBBI", m, 8) == (0, 64, 52, 11, 0, 52, 1023)
            return "<f8", size
        if cls == 0:
            assert m[1] == 0x08
            return {4: "<i4", 8: "<i8"}[size], size
        assert cls == 3
        return "S", size

    @staticmethod
    def dspace(m):
        assert m[0] == 1
        return tuple(struct.unpack_from("<Q", m, 8 + 8 * i)[0] for i in range(m[1]))

    def dataset(self, path):
        msgs = dict(self.header(self.resolve(path)))
        dt, esz = self.dtype(msgs[0x3])
        dims = self.dspace(msgs[0x1])
        lay = msgs[0x8]
        assert lay[0] == 3
        n = int(np.prod(dims)) if dims else 1
        if lay[1] == 1:
            addr, size = struct.unpack_from("<QQ", lay, 2)
            assert size == n * esz
            return np.frombuffer(self.b[addr:addr + size], dtype=dt).reshape(dims)
        assert lay[1] == 2 and 0xB in msgs
        nd = lay[2]
        bt = struct.unpack_from("<Q", lay, 3)[0]
        cdims = struct.unpack_from("<" + "I" * nd, lay, 11)
        assert cdims[-1] == esz and cdims[1:-1] == dims[1:]
        assert self.b[bt:bt + 4] == b"TREE" and self.b[bt + 4] == 1
        used = self.u("H", bt + 6)[0]
        key = 8 + 8 * nd
        out = np.zeros(dims, dtype=dt)
        for i in range(used):
            k = bt + 24 + i * (key + 8)
            size, mask = self.u("II", k)
            r0 = self.u("Q", k + 8)[0]
            child = self.u("Q", k + key)[0]
            assert mask == 0
            raw = zlib.decompress(self.b[child:child + size])
            chunk = np.frombuffer(raw, dtype=dt).reshape((cdims[0],) + dims[1:])
            r1 = min(dims[0], r0 + cdims[0])
            out[r0:r1] = chunk[:r1 - r0]
        return out

    def attrs(self, path):
        out = {}
        for t, m in self.header(self.resolve(path)):
            if t != 0xC:
                continue
            assert m[0] == 1
            nsz, tsz, ssz = struct.unpack_from("<HHH", m, 2)
            r8 = lambda x: (x + 7) // 8 * 8
            name = m[8:8 + nsz - 1].decode()
            p = 8 + r8(nsz)
            dt, esz = self.dtype(m[p:p + tsz])
            p += r8(tsz)
            assert self.dspace(m[p:p + ssz]) == ()
            p += r8(ssz)
            v = m[p:p + esz]
            out[name] = v.rstrip(b"\0").decode() if dt == "S" else np.frombuffer(v, dtype=dt)[0]
        return out


# ---------------------------------------------------------------- generic subset
def test_generic_roundtrip_and_independent_parse(tmp_path):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((37, 5))
    big = rng.standard_normal((300, 41))
    ints = rng.integers(-2**40, 2**40, size=(6, 4))
    i32 = np.arange(-5, 7, dtype=np.int32)
    p = tmp_path / "g.h5"
    with h5io.H5Writer(p) as w:
        w.dataset("/a", a)
        w.dataset("/x/y/big", big, gzip=6)
        w.dataset("/x/ints", ints)
        w.dataset("/x/i32", i32)
        w.dataset("/s", np.float64(2.5))
        w.dataset("/empty", np.zeros((0, 3)))
        w.group("/grp")
        w.attr("/grp", "pi", 3.141592653589793)
        w.attr("/grp", "n", -12)
        w.attr("/grp", "text", "hello, world")
        w.attr("/grp", "blank", "")
        w.attr("/x/y/big", "unit", "bohr")
        for i in range(19):                       # several symbol-table nodes in one group
            w.dataset(f"/many/d{i:02d}", np.array([float(i)]))
    assert not any(n.startswith("g.h5.tmp") for n in os.listdir(tmp_path))
    W = Walk(p)
    np.testing.assert_array_equal(W.dataset("/a"), a)
    np.testing.assert_array_equal(W.dataset("/x/y/big"), big)
    np.testing.assert_array_equal(W.dataset("/x/ints"), ints)
    np.testing.assert_array_equal(W.dataset("/x/i32"), i32)
    assert W.dataset("/s") == 2.5
    assert W.attrs("/grp") == {"pi": 3.141592653589793, "n": -12, "text": "hello, world", "blank": ""}
    assert W.attrs("/x/y/big") == {"unit": "bohr"}
    assert sorted(W.links(W.resolve("/many"))) == [f"d{i:02d}" for i in range(19)]
    with h5io.H5Reader(p) as r:
        assert r.kind("/x") == "group" and r.kind("/a") == "dataset" and r.kind("/nope") == "absent"
        assert r.list("/") == ["a", "empty", "grp", "many", "s", "x"]
        np.testing.assert_array_equal(r.read("/a"), a)
        np.testing.assert_array_equal(r.read("/x/y/big"), big)
        np.testing.assert_array_equal(r.read("/x/y/big", start=(123, 7), count=(100, 30)), big[123:223, 7:37])
        np.testing.assert_array_equal(r.read("/a", start=(3, 1), count=(2, 3)), a[3:5, 1:4])
        np.testing.assert_array_equal(r.read("/x/ints"), ints)
        assert r.read("/x/i32").dtype == np.int64
        np.testing.assert_array_equal(r.read("/x/i32"), i32)
        assert r.read("/s") == 2.5
        assert r.shape("/empty") == ((0, 3), "float")
        assert r.attr("/grp", "pi") == 3.141592653589793
        assert r.attr("/grp", "n") == -12
        assert r.attr("/grp", "text") == "hello, world"
        assert r.attr("/x/y/big", "unit") == "bohr"
        with pytest.raises(KeyError):
            r.attr("/grp", "missing")
        with pytest.raises(_lib.ScattError) as e:
            r.read("/a", start=(30, 0), count=(10, 5))       # outside the dataset
        assert e.value.code == 11


def test_missing_and_foreign_files_are_io_errors(tmp_path):
    with pytest.raises(_lib.ScattError) as e:
        h5io.H5Reader(tmp_path / "absent.h5")
    assert e.value.code == 11
    junk = tmp_path / "junk.h5"
    junk.write_bytes(b"not an hdf5 file" * 64)
    with pytest.raises(_lib.ScattError) as e:
        h5io.H5Reader(junk)
    assert e.value.code == 11
    with pytest.raises(_lib.ScattError) as e:
        h5io.Preproc(junk)
    assert e.value.code == 11


def test_writer_discards_on_error(tmp_path):
    p = tmp_path / "d.h5"
    with pytest.raises(RuntimeError):
        with h5io.H5Writer(p) as w:
            w.dataset("/a", np.ones(3))
            raise RuntimeError("abandon")
    assert os.listdir(tmp_path) == []


# ---------------------------------------------------------------- dipole scan output
def fake_result(n, no, seed):
    rng = np.random.default_rng(seed)
    c = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    return types.SimpleNamespace(
        A=rng.standard_normal((n, n)), B=rng.standard_normal((n, n)), b_overlap=rng.standard_normal((n, no)),
        D=c(6, n), D_raw=c(6, n), d_raw=rng.standard_normal((6, n)), d_corr=rng.standard_normal((6, no)),
        partial_sigma=rng.random(6), diag={"fit_residual_rel": 1e-9 * seed, "K_symmetry_err_aa": 3e-13})


def test_dipole_scan_layout(tmp_path):
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)
    meta = h5io.scan_meta(inp, dk=0.05, ik_min=1, ik_max=41, molecule_name="h2o_like", iso_date_utc="2026-01-01T00:00:00Z")
    res = [(7, fake_result(16, 3, 1)), (12, fake_result(16, 3, 2))]
    d = tmp_path / "scan"
    assert h5io.write_dipole_scan(d, meta, res) == [7, 12]
    assert sorted(os.listdir(d)) == ["__SUCCESS__", "ik0007.h5", "ik0012.h5", "manifest.h5"]
    W = Walk(d / "manifest.h5")
    g = W.attrs("/grid")
    assert g["dr"] == 0.05 and g["N_grid"] == 301 and g["l_max_continuum"] == 3 and g["r_min"] == 0.0
    assert g["E_HOMO"] == inp.orb_energies[inp.n_occ - 1]
    assert W.attrs("/kgrid") == {"dk": 0.05, "ik_min": 1, "ik_max": 41}
    np.testing.assert_array_equal(W.dataset("/occ/energies"), inp.orb_energies[:inp.n_occ])
    np.testing.assert_array_equal(W.dataset("/occ/spin_factors"), np.full(inp.n_occ, 2.0))
    np.testing.assert_array_equal(W.dataset("/atoms/Z"), inp.atoms[:, 0].astype(int))
    np.testing.assert_array_equal(W.dataset("/atoms/xyz_bohr"), inp.atoms[:, 1:])
    assert W.attrs("/conventions")["real_Ylm_q_map"] == "x=+1, y=-1, z=0"
    assert W.attrs("/run")["molecule_name"] == "h2o_like"
    E = Walk(d / "ik0012.h5")
    m = E.attrs("/meta")
    k = 12 * 0.05
    assert m["ik"] == 12 and m["k"] == k and m["E"] == 0.5 * k * k
    assert m["omega"] == 0.5 * k * k - g["E_HOMO"]
    assert m["fit_residual_rel"] == 2e-9 and m["K_symmetry_err"] == 3e-13
    r = res[1][1]
    np.testing.assert_array_equal(E.dataset("/A"), r.A)
    np.testing.assert_array_equal(E.dataset("/b_overlap"), r.b_overlap)
    for s, (gg, p) in enumerate(h5io.DipoleReader.SLICES):
        b = f"/dipole/{gg}/{p}/"
        np.testing.assert_array_equal(E.dataset(b + "D_ortho_im"), r.D[s].imag)
        np.testing.assert_array_equal(E.dataset(b + "D_raw_re"), r.D_raw[s].real)
        np.testing.assert_array_equal(E.dataset(b + "d_correction"), r.d_corr[s])
        assert E.attrs(b[:-1])["partial_sigma"] == r.partial_sigma[s]
    rd = h5io.DipoleReader(d)
    assert rd.available_ik() == [7, 12]
    back = rd.read_energy(7)
    np.testing.assert_array_equal(back["B"], res[0][1].B)
    np.testing.assert_array_equal(back["slices"][4]["D"], res[0][1].D[4])
    assert rd.meta["molecule_name"] == "h2o_like" and rd.meta["ik_max"] == 41
    # resume: existing energies are skipped, the manifest is kept
    m0 = os.path.getmtime(d / "manifest.h5")
    assert h5io.write_dipole_scan(d, meta, res + [(13, fake_result(16, 3, 3))]) == [13]
    assert os.path.getmtime(d / "manifest.h5") == m0


def test_dipole_meta_validation(tmp_path):
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=3)
    with pytest.raises(_lib.ScattError) as e:
        h5io.write_dipole_scan(tmp_path / "s", h5io.scan_meta(inp, dk=0.0, ik_min=1, ik_max=5), [])
    assert e.value.code == 1


# ---------------------------------------------------------------- preprocessing input
@pytest.mark.parametrize("split", [False, True])
def test_preproc_roundtrip(tmp_path, split):
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=11, lmax_orb=8, n_orb=2)
    path = h5io.write_preproc(tmp_path / "h2o", inp, split=split)
    if split:
        assert sorted(os.listdir(tmp_path)) == ["h2o.orbitals.h5", "h2o.potentials.h5"]
        # either sibling opens the pair
        h5io.Preproc(str(tmp_path / "h2o.potentials.h5")).close()
    W = Walk(path)
    assert W.dataset("/grid/N") == 301
    with h5io.Preproc(path) as pp:
        assert (pp.Nr, pp.dr, pp.n_occ, pp.n_sce, pp.rmin) == (301, 0.05, inp.n_occ, 2, 0.0)
        assert not pp.has_initial_state
        np.testing.assert_array_equal(pp.orb_energies, inp.orb_energies)
        for l in (3, 11):
            d, E_init = pp.desc(l)
            assert E_init == inp.orb_energies[inp.n_occ - 1]
            cut = min((l + min(l, 10) + 1) ** 2, inp.psi_lm.shape[1])
            psi, vh = pp.arrays(d)
            assert (d.n_orb, d.Nlm_store, d.Nr_store, d.init_state) == (2, cut, inp.psi_lm.shape[2], -1)
            np.testing.assert_array_equal(psi, inp.psi_lm[:, :cut])
            assert d.n_H == min(pp.Nlm_orb_store, (2 * l + 1) ** 2)
            np.testing.assert_array_equal(vh[:inp.V_H.shape[0]], inp.V_H)
            assert not vh[inp.V_H.shape[0]:].any()
            np.testing.assert_array_equal(pp.atoms, inp.atoms)
            assert (d.n_occ, d.l_cont_max, d.alpha_pol) == (inp.n_occ, l, 0.0)


def test_preproc_initial_state_becomes_last_orbital(tmp_path):
    inp = synth.h2_like(Nr=401, dr=0.05, l_cont=3)
    rng = np.random.default_rng(3)
    init = rng.standard_normal((30, inp.psi_lm.shape[2]))
    path = h5io.write_preproc(tmp_path / "a.h5", inp, initial_state=(init, -0.12, 1.0))
    with h5io.Preproc(path) as pp:
        assert pp.has_initial_state and pp.E_init == -0.12
        d, E_init = pp.desc(3)
        assert E_init == -0.12
        psi, _ = pp.arrays(d)
        assert d.n_orb == inp.psi_lm.shape[0] + 1 and d.init_state == inp.psi_lm.shape[0]
        cut = (3 + 3 + 1) ** 2
        assert d.Nlm_store == max(min(cut, inp.psi_lm.shape[1]), min(cut, 30))
        np.testing.assert_array_equal(psi[-1, :min(cut, 30)], init[:min(cut, 30)])
        assert not psi[-1, min(cut, 30):].any()


def test_cpp_interface(tmp_path):
    """host/scatt_io.hpp compiled against the library: DipoleWriter ->
    DipoleReader bit for bit, HDF5Reader on a file written here."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "spion-emol_b200")
    exe = tmp_path / "host_io_check"
    cmd = ["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
           "-I", os.path.join(pkg, "host"), os.path.join(root, "tests", "host_io_check.cpp"), "-o", str(exe),
           "-L", pkg, "-lscatt_b200", f"-Wl,-rpath,{pkg}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    inp = synth.h2o_like(Nr=301, dr=0.05, l_cont=3, lmax_orb=6, n_orb=3)
    pre = h5io.write_preproc(tmp_path / "m", inp, split=True)
    r = subprocess.run([str(exe), str(tmp_path / "scan"), pre], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l.split() for l in r.stdout.splitlines()]
    assert lines[0] == ["dipole", "ok"]
    pre_line, desc = lines[1], lines[2]
    assert pre_line[1] == "301" and pre_line[4] == str(inp.n_occ) and pre_line[5] == "3"
    assert float(pre_line[10]) == 0.05 and float(pre_line[11]) == inp.orb_energies[-1]
    cut = min((3 + 3 + 1) ** 2, inp.psi_lm.shape[1])
    assert desc[1:5] == ["3", str(cut), str(inp.psi_lm.shape[2]), "-1"]
    assert float(desc[8]) == inp.psi_lm[0, 0, 1]
    assert float(desc[9]) == inp.orb_energies[inp.n_occ - 1]


def test_preproc_extra_datasets(tmp_path):
    """The density and the local exchange the preprocessing chain computes
    land beside V_H (main_preprocess.cpp:706-714) and read back unchanged."""
    inp = synth.h2_like(Nr=101, dr=0.1, l_cont=2)
    rng = np.random.default_rng(5)
    rho, vx = rng.standard_normal((9, 101)), rng.standard_normal((9, 101))
    path = h5io.write_preproc(tmp_path / "x.h5", inp,
                              extra={"/rho/rho_lm": rho, "/potential/V_local_exchange": vx})
    with h5io.H5Reader(path) as r:
        np.testing.assert_array_equal(r.read("/rho/rho_lm"), rho)
        np.testing.assert_array_equal(r.read("/potential/V_local_exchange"), vx)
    with h5io.Preproc(path) as pp:
        assert pp.Nr == 101

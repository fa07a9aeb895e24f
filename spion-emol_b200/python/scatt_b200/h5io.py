"""Files around the path, through the library's HDF5 subset (no libhdf5, no h5py).

* H5Writer / H5Reader: generic groups, datasets and scalar attributes.
* Dipole scan output in the reference's DipoleWriter layout
  (src/scatt/DipoleIO.hpp:115-148, DipoleIO.cpp:141-336): scan_meta,
  write_dipole_scan, DipoleReader.
* Preprocessing input in the reference's HDF5Reader schema
  (src/io/HDF5Reader.hpp:42-86, 446-570): write_preproc (from synthetic
  inputs) and Preproc (what scatt_preproc_* reads back).

All of it is host code in libscatt_b200.so; nothing here needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import ScattError, as_dptr, check, lib

cp = C.c_char_p
vp = C.c_void_p
ll = C.c_longlong
llp = C.POINTER(C.c_longlong)


class DipoleMeta(C.Structure):
    _fields_ = [("r_min", C.c_double), ("dr", C.c_double), ("N_grid", ll), ("l_max_continuum", C.c_int),
                ("dk", C.c_double), ("ik_min", C.c_int), ("ik_max", C.c_int), ("E_HOMO", C.c_double),
                ("n_occ", C.c_int), ("occ_energies", C.POINTER(C.c_double)),
                ("occ_spin_factors", C.POINTER(C.c_double)), ("n_atoms", C.c_int),
                ("Z", C.POINTER(C.c_int)), ("xyz_bohr", C.POINTER(C.c_double)),
                ("molecule_name", cp), ("git_hash", cp), ("iso_date_utc", cp), ("psi_dir_prefix", cp)]


class DipoleEnergy(C.Structure):
    _fields_ = [("ik", C.c_int), ("n_ch", C.c_int), ("n_occ", C.c_int),
                ("A", C.POINTER(C.c_double)), ("B", C.POINTER(C.c_double)),
                ("b_overlap", C.POINTER(C.c_double)),
                ("D_re", C.POINTER(C.c_double)), ("D_im", C.POINTER(C.c_double)),
                ("Draw_re", C.POINTER(C.c_double)), ("Draw_im", C.POINTER(C.c_double)),
                ("d_raw", C.POINTER(C.c_double)), ("d_corr", C.POINTER(C.c_double)),
                ("partial_sigma", C.POINTER(C.c_double)),
                ("fit_residual_rel", C.c_double), ("K_symmetry_err", C.c_double)]


_bound = False


def _bind():
    global _bound
    if _bound:
        return
    L = lib()
    vpp = C.POINTER(vp)
    L.scatt_h5w_open.argtypes = [cp, vpp]
    L.scatt_h5w_group.argtypes = [vp, cp]
    L.scatt_h5w_dataset.argtypes = [vp, cp, C.c_int, C.c_int, llp, vp, C.c_int]
    L.scatt_h5w_attr_f64.argtypes = [vp, cp, cp, C.c_double]
    L.scatt_h5w_attr_i64.argtypes = [vp, cp, cp, ll]
    L.scatt_h5w_attr_str.argtypes = [vp, cp, cp, cp]
    L.scatt_h5w_close.argtypes = [vp, C.c_int]
    L.scatt_h5r_open.argtypes = [cp, vpp]
    L.scatt_h5r_kind.argtypes = [vp, cp, C.POINTER(C.c_int)]
    L.scatt_h5r_shape.argtypes = [vp, cp, C.POINTER(C.c_int), llp, C.POINTER(C.c_int)]
    L.scatt_h5r_read.argtypes = [vp, cp, C.c_int, C.c_int, llp, llp, vp]
    L.scatt_h5r_list.argtypes = [vp, cp, C.c_char_p, ll, llp]
    L.scatt_h5r_attr.argtypes = [vp, cp, cp, C.POINTER(C.c_int), C.POINTER(C.c_double), llp, C.c_char_p, ll]
    L.scatt_h5r_close.argtypes = [vp]
    L.scatt_dipole_open.argtypes = [cp, C.POINTER(DipoleMeta)]
    L.scatt_dipole_has_energy.argtypes = [cp, C.c_int, C.POINTER(C.c_int)]
    L.scatt_dipole_write_energy.argtypes = [cp, C.POINTER(DipoleMeta), C.POINTER(DipoleEnergy)]
    L.scatt_dipole_finalize.argtypes = [cp]
    L.scatt_preproc_open.argtypes = [cp, vpp]
    L.scatt_preproc_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.scatt_preproc_orbital_energies.argtypes = [vp, C.POINTER(C.c_double), C.c_int]
    L.scatt_preproc_atoms.argtypes = [vp, C.POINTER(C.c_double), C.c_int]
    L.scatt_preproc_desc.argtypes = [vp, C.c_int, vp, C.POINTER(C.c_double)]
    L.scatt_preproc_close.argtypes = [vp]
    _bound = True


def _b(s: str) -> bytes:
    return s.encode()


def _lls(seq):
    a = (ll * max(len(seq), 1))()
    for i, v in enumerate(seq):
        a[i] = int(v)
    return a


# ---------------------------------------------------------------- generic
class H5Writer:
    """with H5Writer(path) as w: w.dataset("/g/x", array); w.attr("/g", "n", 3)
    The file appears at `path` when the block ends without an exception."""

    def __init__(self, path: str):
        _bind()
        self.h = vp()
        check(lib().scatt_h5w_open(_b(os.fspath(path)), C.byref(self.h)))

    def group(self, path: str):
        check(lib().scatt_h5w_group(self.h, _b(path)))

    def dataset(self, path: str, data, gzip: int = 0):
        a = np.asarray(data)
        if a.dtype.kind == "f":
            a, kind = np.ascontiguousarray(a, dtype=np.float64), 0
        elif a.dtype == np.int32:
            a, kind = np.ascontiguousarray(a), 2
        elif a.dtype.kind in "iub":
            a, kind = np.ascontiguousarray(a, dtype=np.int64), 1
        else:
            raise TypeError(f"{path}: dtype {a.dtype} is not written")
        check(lib().scatt_h5w_dataset(self.h, _b(path), kind, a.ndim, _lls(a.shape),
                                      a.ctypes.data_as(vp), int(gzip)))

    def attr(self, obj: str, name: str, value):
        if isinstance(value, str):
            check(lib().scatt_h5w_attr_str(self.h, _b(obj), _b(name), _b(value)))
        elif isinstance(value, (bool, int, np.integer)):
            check(lib().scatt_h5w_attr_i64(self.h, _b(obj), _b(name), int(value)))
        else:
            check(lib().scatt_h5w_attr_f64(self.h, _b(obj), _b(name), float(value)))

    def close(self, keep: bool = True):
        if self.h:
            h, self.h = self.h, vp()
            check(lib().scatt_h5w_close(h, 1 if keep else 0))

    def __enter__(self):
        return self

    def __exit__(self, et, ev, tb):
        self.close(keep=et is None)


class H5Reader:
    def __init__(self, path: str):
        _bind()
        self.h = vp()
        check(lib().scatt_h5r_open(_b(os.fspath(path)), C.byref(self.h)))

    def kind(self, path: str) -> str:
        k = C.c_int(0)
        check(lib().scatt_h5r_kind(self.h, _b(path), C.byref(k)))
        return ("absent", "group", "dataset")[k.value]

    def exists(self, path: str) -> bool:
        return self.kind(path) != "absent"

    def shape(self, path: str):
        rank, ek = C.c_int(0), C.c_int(0)
        dims = (ll * 8)()
        check(lib().scatt_h5r_shape(self.h, _b(path), C.byref(rank), dims, C.byref(ek)))
        return tuple(dims[i] for i in range(rank.value)), ("float", "int", None, "str")[ek.value]

    def read(self, path: str, start=None, count=None):
        """The dataset (or the block [start, start + count)), as float64 or int64."""
        dims, ek = self.shape(path)
        as_int = ek == "int"
        shp = tuple(count) if count is not None else dims
        out = np.empty(shp, dtype=np.int64 if as_int else np.float64)
        st = _lls(start) if start is not None else None
        ct = _lls(count) if count is not None else None
        check(lib().scatt_h5r_read(self.h, _b(path), 1 if as_int else 0, len(dims), st, ct, out.ctypes.data_as(vp)))
        return out

    def list(self, group: str = "/"):
        need = ll(0)
        check(lib().scatt_h5r_list(self.h, _b(group), None, 0, C.byref(need)))
        buf = C.create_string_buffer(int(need.value))
        check(lib().scatt_h5r_list(self.h, _b(group), buf, need.value, None))
        return [x for x in buf.value.decode().split("\n") if x]

    def attr(self, obj: str, name: str):
        k, f, i = C.c_int(0), C.c_double(0.0), ll(0)
        buf = C.create_string_buffer(4096)
        check(lib().scatt_h5r_attr(self.h, _b(obj), _b(name), C.byref(k), C.byref(f), C.byref(i), buf, 4096))
        if k.value == 0:
            raise KeyError(f"{obj}:{name}")
        return {1: f.value, 2: i.value, 3: buf.value.decode()}[k.value]

    def close(self):
        if self.h:
            lib().scatt_h5r_close(self.h)
            self.h = vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- dipole scan output
class ScanMeta:
    """scatt_dipole_meta with the arrays it points at kept alive."""

    def __init__(self, *, dr, N_grid, l_max_continuum, dk, ik_min, ik_max, E_HOMO, occ_energies=(),
                 occ_spin_factors=None, atoms=None, r_min=0.0, molecule_name="", git_hash="",
                 iso_date_utc="", psi_dir_prefix=""):
        self.occ_e = np.ascontiguousarray(occ_energies, dtype=np.float64)
        self.occ_s = (np.full(self.occ_e.size, 2.0) if occ_spin_factors is None
                      else np.ascontiguousarray(occ_spin_factors, dtype=np.float64))
        at = np.zeros((0, 4)) if atoms is None else np.asarray(atoms, dtype=np.float64).reshape(-1, 4)
        self.Z = np.ascontiguousarray(np.rint(at[:, 0]).astype(np.int32))
        self.xyz = np.ascontiguousarray(at[:, 1:4])
        self.strings = [_b(s) for s in (molecule_name, git_hash, iso_date_utc, psi_dir_prefix)]
        m = DipoleMeta()
        m.r_min, m.dr, m.N_grid, m.l_max_continuum = float(r_min), float(dr), int(N_grid), int(l_max_continuum)
        m.dk, m.ik_min, m.ik_max, m.E_HOMO = float(dk), int(ik_min), int(ik_max), float(E_HOMO)
        m.n_occ = self.occ_e.size
        m.occ_energies, m.occ_spin_factors = as_dptr(self.occ_e), as_dptr(self.occ_s)
        m.n_atoms = self.Z.size
        m.Z = self.Z.ctypes.data_as(C.POINTER(C.c_int))
        m.xyz_bohr = as_dptr(self.xyz)
        m.molecule_name, m.git_hash, m.iso_date_utc, m.psi_dir_prefix = self.strings
        self.c = m


def scan_meta(inp, dk, ik_min, ik_max, E_HOMO=None, **kw) -> ScanMeta:
    """The manifest of a scan over the k grid ik * dk (ik_min <= ik < ik_max)
    of the inputs `inp` (synthetic ScanInputs or a Preproc)."""
    occ = np.asarray(inp.orb_energies[:inp.n_occ], dtype=np.float64)
    if E_HOMO is None:
        E_HOMO = float(occ[-1])
    return ScanMeta(dr=inp.dr, N_grid=inp.Nr, l_max_continuum=inp.l_cont, dk=dk, ik_min=ik_min, ik_max=ik_max,
                    E_HOMO=E_HOMO, occ_energies=occ, atoms=inp.atoms,
                    molecule_name=kw.pop("molecule_name", getattr(inp, "name", "")), **kw)


def energy_payload(ik, r):
    """scatt_dipole_energy of one EnergyResult (arrays kept on the returned object)."""
    n = r.A.shape[0]
    arrs = {
        "A": np.ascontiguousarray(r.A), "B": np.ascontiguousarray(r.B),
        "b_overlap": np.ascontiguousarray(r.b_overlap),
        "D_re": np.ascontiguousarray(np.real(r.D)), "D_im": np.ascontiguousarray(np.imag(r.D)),
        "Draw_re": np.ascontiguousarray(np.real(r.D_raw)), "Draw_im": np.ascontiguousarray(np.imag(r.D_raw)),
        "d_raw": np.ascontiguousarray(r.d_raw), "d_corr": np.ascontiguousarray(r.d_corr),
        "partial_sigma": np.ascontiguousarray(r.partial_sigma),
    }
    e = DipoleEnergy()
    e.ik, e.n_ch, e.n_occ = int(ik), n, arrs["b_overlap"].shape[1]
    for k, v in arrs.items():
        assert v.dtype == np.float64
        setattr(e, k, as_dptr(v))
    e.fit_residual_rel = float(r.diag.get("fit_residual_rel", 0.0))
    e.K_symmetry_err = float(r.diag.get("K_symmetry_err_aa", 0.0))
    e._keep = arrs
    return e


def write_dipole_scan(scan_dir, meta: ScanMeta, results, finalize=True, skip_existing=True):
    """Writes manifest.h5 (when absent) and ik<NNNN>.h5 for each (ik,
    EnergyResult); existing energy files are skipped (a resumed scan)."""
    _bind()
    d = _b(os.fspath(scan_dir))
    check(lib().scatt_dipole_open(d, C.byref(meta.c)))
    written = []
    for ik, r in results:
        has = C.c_int(0)
        check(lib().scatt_dipole_has_energy(d, int(ik), C.byref(has)))
        if has.value and skip_existing:
            continue
        e = energy_payload(ik, r)
        check(lib().scatt_dipole_write_energy(d, C.byref(meta.c), C.byref(e)))
        written.append(int(ik))
    if finalize:
        check(lib().scatt_dipole_finalize(d))
    return written


class DipoleReader:
    """Read-back of a dipole scan directory (the reference's DipoleReader,
    src/scatt/DipoleIO.hpp:160-176)."""

    SLICES = [(g, p) for g in ("length", "velocity") for p in ("x", "y", "z")]

    def __init__(self, scan_dir):
        self.dir = os.fspath(scan_dir)
        with H5Reader(os.path.join(self.dir, "manifest.h5")) as h:
            m = {k: h.attr("/grid", k) for k in ("r_min", "dr", "N_grid", "l_max_continuum", "E_HOMO")}
            m.update({k: h.attr("/kgrid", k) for k in ("dk", "ik_min", "ik_max")})
            if h.exists("/occ"):
                m["occ_energies"] = h.read("/occ/energies")
                m["occ_spin_factors"] = h.read("/occ/spin_factors")
            if h.exists("/atoms"):
                m["Z"] = h.read("/atoms/Z")
                m["xyz_bohr"] = h.read("/atoms/xyz_bohr")
            for k in ("molecule_name", "git_hash", "iso_date_utc", "psi_dir_prefix"):
                m[k] = h.attr("/run", k)
        self.meta = m

    def available_ik(self):
        out = []
        for n in os.listdir(self.dir):
            if n.startswith("ik") and n.endswith(".h5") and n[2:-3].isdigit():
                out.append(int(n[2:-3]))
        return sorted(out)

    def read_energy(self, ik):
        tag = "ik" + str(int(ik)).zfill(4)
        with H5Reader(os.path.join(self.dir, tag + ".h5")) as h:
            r = {k: h.attr("/meta", k) for k in ("ik", "k", "E", "omega", "fit_residual_rel", "K_symmetry_err")}
            for k in ("A", "B", "b_overlap"):
                r[k] = h.read("/" + k)
            sl = []
            for g, p in self.SLICES:
                b = f"/dipole/{g}/{p}/"
                sl.append({"D": h.read(b + "D_ortho_re") + 1j * h.read(b + "D_ortho_im"),
                           "D_raw": h.read(b + "D_raw_re") + 1j * h.read(b + "D_raw_im"),
                           "d_raw": h.read(b + "d_raw"), "d_corr": h.read(b + "d_correction"),
                           "partial_sigma": h.attr(f"/dipole/{g}/{p}", "partial_sigma")})
            r["slices"] = sl
        return r


# ---------------------------------------------------------------- preprocessing input
def _isqrt_ceil(n):
    r = int(np.sqrt(n))
    while r * r < n:
        r += 1
    return r


def write_preproc(path, inp, split=False, gzip=4, initial_state=None, extra=None):
    """Writes the energy-independent inputs `inp` in the reference's
    preprocessing schema (combined file at `path`, or with split=True the
    pair <stem>.orbitals.h5 + <stem>.potentials.h5 where path is the stem).
    initial_state = (psi (Nlm, Nr_store), energy, occupation) adds the
    /initial_state group; extra = {dataset path: array} adds datasets to
    the potentials side (e.g. /potential/V_local_exchange and /rho/rho_lm,
    main_preprocess.cpp:706-714).  Returns the path to open."""
    psi = np.asarray(inp.psi_lm, dtype=np.float64)
    n_orb, Nlm, Nr_store = psi.shape
    L = _isqrt_ceil(max(Nlm, inp.V_H.shape[0])) - 1
    Nlm_sce = (L + 1) ** 2
    vh = np.zeros((Nlm_sce, inp.Nr))
    vh[:inp.V_H.shape[0]] = inp.V_H
    psi_rows = np.zeros((n_orb, Nlm_sce, Nr_store))
    psi_rows[:, :Nlm] = psi
    occ = np.where(np.arange(n_orb) < inp.n_occ, 2.0, 0.0)
    at = np.asarray(inp.atoms, dtype=np.float64).reshape(-1, 4)

    def shared(w):
        w.dataset("/grid/rmin", np.float64(0.0))
        w.dataset("/grid/dr", np.float64(inp.dr))
        w.dataset("/grid/N", np.int64(inp.Nr))
        w.dataset("/angular/Lmax", np.int64(L))
        w.dataset("/geometry/Z", np.rint(at[:, 0]).astype(np.int32))
        w.dataset("/geometry/xyz_bohr", at[:, 1:4])

    def orbitals(w):
        w.dataset("/orbitals/n_alpha", np.int64(n_orb))
        w.dataset("/orbitals/n_occ_alpha", np.int64(inp.n_occ))
        w.dataset("/orbitals/n_sce", np.int64(n_orb))
        w.dataset("/orbitals/Lmax_orb_store", np.int64(L))
        w.dataset("/orbitals/Nlm_orb_store", np.int64(Nlm_sce))
        w.dataset("/orbitals/Nr_orb_store", np.int64(Nr_store))
        w.dataset("/orbitals/psi_lm", psi_rows.reshape(n_orb * Nlm_sce, Nr_store), gzip=gzip)
        w.dataset("/orbitals/energies_hartree", np.asarray(inp.orb_energies, dtype=np.float64))
        w.dataset("/orbitals/occupations", occ)
        w.dataset("/orbitals/molden_index", np.arange(1, n_orb + 1, dtype=np.int32))
        if initial_state is not None:
            ip, ie, io = initial_state
            w.dataset("/initial_state/psi_lm", np.asarray(ip, dtype=np.float64), gzip=gzip)
            w.dataset("/initial_state/energy_hartree", np.float64(ie))
            w.dataset("/initial_state/occupation", np.float64(io))

    def potentials(w):
        w.dataset("/potential/V_H", vh, gzip=gzip)
        if inp.alpha_pol > 0:
            w.dataset("/polarizability/alpha_tensor", np.eye(3) * inp.alpha_pol)
            w.dataset("/polarizability/alpha_iso_au", np.float64(inp.alpha_pol))
        w.dataset("/meta/schema_version", np.int64(2))
        for name, arr in (extra or {}).items():
            w.dataset(name, np.asarray(arr, dtype=np.float64), gzip=gzip)

    path = os.fspath(path)
    if not split:
        with H5Writer(path) as w:
            shared(w)
            orbitals(w)
            potentials(w)
        return path
    orb, pot = path + ".orbitals.h5", path + ".potentials.h5"
    with H5Writer(orb) as w:
        shared(w)
        orbitals(w)
    with H5Writer(pot) as w:
        shared(w)
        potentials(w)
    return orb


class Preproc:
    """A preprocessing file opened through scatt_preproc_* (split or combined
    layout, detected as the reference's HDF5Reader does)."""

    def __init__(self, path):
        _bind()
        self.h = vp()
        check(lib().scatt_preproc_open(_b(os.fspath(path)), C.byref(self.h)))
        iv = (C.c_int * 8)()
        dv = (C.c_double * 4)()
        check(lib().scatt_preproc_info(self.h, iv, dv))
        (self.Nr, self.Lmax_sce, self.n_alpha, self.n_occ, self.n_sce, self.Nlm_orb_store,
         self.Nr_orb_store, hi) = list(iv)
        self.has_initial_state = bool(hi)
        self.rmin, self.dr, self.E_init, self.alpha_iso = list(dv)
        e = np.zeros(self.n_sce)
        check(lib().scatt_preproc_orbital_energies(self.h, as_dptr(e), e.size))
        self.orb_energies = e
        self.atoms = np.zeros((0, 4))

    def desc(self, l_cont_max):
        """(ScanDesc, E_init): valid until the next desc() or close()."""
        from .solver import ScanDesc
        d = ScanDesc()
        E = C.c_double(0.0)
        check(lib().scatt_preproc_desc(self.h, int(l_cont_max), C.cast(C.byref(d), vp), C.byref(E)))
        na = d.n_atoms
        a = np.zeros((na, 4))
        if na:
            check(lib().scatt_preproc_atoms(self.h, as_dptr(a), na))
        self.atoms = a
        return d, E.value

    def arrays(self, d):
        """Copies of what a desc points at: psi_lm (n_orb, Nlm, Nr_store), V_H (n_H, Nr)."""
        psi = np.ctypeslib.as_array(d.psi_lm, shape=(d.n_orb * d.Nlm_store * d.Nr_store,)).copy()
        vh = np.ctypeslib.as_array(d.V_H, shape=(d.n_H * d.Nr,)).copy()
        return psi.reshape(d.n_orb, d.Nlm_store, d.Nr_store), vh.reshape(d.n_H, d.Nr)

    def close(self):
        if self.h:
            lib().scatt_preproc_close(self.h)
            self.h = vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["H5Writer", "H5Reader", "ScanMeta", "scan_meta", "write_dipole_scan", "DipoleReader",
           "write_preproc", "Preproc", "ScattError"]

"""The reference's on-disk psi store (scatt_psi_store_*: PotentialStorage
chunks, metadata.bin, psi_asym.bin, manifest.txt, __SUCCESS__), written from
ScanSolver.psi_sweep's output and read back, e.g. for the
continuum-continuum dipole (scatt_b200._lib.cc_dipole)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import as_dptr, check, dptr, lib


class StoreMeta(C.Structure):
    _fields_ = [("energy", C.c_double), ("dr", C.c_double)] + [
        (n, C.c_int) for n in ("n_grid", "n_psi", "n_f", "l_cont", "l_exch", "n_occ", "n_transition", "keep_lo",
                               "keep_hi", "chunk_size", "n_asym", "asym_offset")]


_bound = False


def _bind():
    global _bound
    if _bound:
        return
    L = lib()
    vp = C.c_void_p
    L.scatt_psi_store_dirname.argtypes = [C.POINTER(StoreMeta), C.c_char_p, C.c_int]
    L.scatt_psi_store_write.argtypes = [C.c_char_p, C.POINTER(StoreMeta), dptr, C.c_int, dptr, C.c_int]
    L.scatt_psi_store_open.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.scatt_psi_store_info.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.scatt_psi_store_manifest.argtypes = [vp, C.c_char_p, C.c_int]
    L.scatt_psi_store_read.argtypes = [vp, C.c_longlong, C.c_longlong, dptr]
    L.scatt_psi_store_read_asym.argtypes = [vp, dptr]
    L.scatt_psi_store_close.argtypes = [vp]
    _bound = True


def meta(**kw) -> StoreMeta:
    m = StoreMeta()
    m.chunk_size = 64
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def dirname(m: StoreMeta) -> str:
    """The reference's default directory name (psi_Nr.._Npsi.._E.._lc.._keep..-..)."""
    _bind()
    buf = C.create_string_buffer(512)
    check(lib().scatt_psi_store_dirname(C.byref(m), buf, 512))
    return buf.value.decode()


def _column_major(a):
    """The C-order buffer of column-major matrices from (n, rows, cols) views
    whose rows are the channels (psi_sweep's output), and its ld."""
    b = np.ascontiguousarray(np.swapaxes(np.asarray(a, dtype=np.float64), -1, -2))
    return b, b.shape[-1]


def write(path, m: StoreMeta, psi, psi_asym=None) -> str:
    """psi: (keep_hi - keep_lo + 1, L, L) with psi[i][:N_psi, :N_psi] the
    point keep_lo + i (rows = channel); psi_asym: (n_asym, L', L') or None."""
    _bind()
    pb, ld = _column_major(psi)
    if pb.shape[0] != m.keep_hi - m.keep_lo + 1:
        raise ValueError("psi must hold keep_hi - keep_lo + 1 points")
    ab, lda = (_column_major(psi_asym) if psi_asym is not None else (None, 0))
    if ab is not None:
        m.n_asym = ab.shape[0]
    check(lib().scatt_psi_store_write(os.fsencode(os.fspath(path)), C.byref(m), as_dptr(pb), int(ld),
                                      as_dptr(ab) if ab is not None else None, int(lda)))
    return os.fspath(path)


class Store:
    """An open store: .points, .n_psi, .chunk_size, .chunks, .n_asym,
    .asym_offset, .manifest; read(first, count) -> (count, N_psi, N_psi)
    with rows = channel; asym() likewise for the asymptotic buffer."""

    def __init__(self, path):
        _bind()
        self.h = C.c_void_p()
        check(lib().scatt_psi_store_open(os.fsencode(os.fspath(path)), C.byref(self.h)))
        info = (C.c_longlong * 6)()
        check(lib().scatt_psi_store_info(self.h, info))
        self.points, self.n_psi, self.chunk_size, self.chunks, self.n_asym, self.asym_offset = (int(x) for x in info)
        buf = C.create_string_buffer(4096)
        check(lib().scatt_psi_store_manifest(self.h, buf, 4096))
        self.manifest = buf.value.decode()

    def read(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.points - first if count is None else count
        out = np.zeros((count, self.n_psi, self.n_psi))
        check(lib().scatt_psi_store_read(self.h, int(first), int(count), as_dptr(out)))
        return np.swapaxes(out, 1, 2)

    def asym(self) -> np.ndarray:
        out = np.zeros((self.n_asym, self.n_psi, self.n_psi))
        check(lib().scatt_psi_store_read_asym(self.h, as_dptr(out)))
        return np.swapaxes(out, 1, 2)

    def close(self):
        if self.h:
            lib().scatt_psi_store_close(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

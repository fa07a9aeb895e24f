"""Molden files through the library's reader (scatt_molden_*: the
[Atoms], [GTO] and [MO] sections of preprocessing/src/molden/Molden.hpp),
in the arrays the device expansion of the basis takes
(scatt_b200._lib.sce_basis)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import as_dptr, as_iptr, check, dptr, iptr, lib

_bound = False


def _bind():
    global _bound
    if _bound:
        return
    L = lib()
    vp = C.c_void_p
    L.scatt_molden_open.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.scatt_molden_info.argtypes = [vp, iptr]
    L.scatt_molden_atoms.argtypes = [vp, dptr]
    L.scatt_molden_shells.argtypes = [vp, iptr, iptr, dptr, dptr, dptr]
    L.scatt_molden_mos.argtypes = [vp, C.c_int, dptr, dptr, dptr]
    L.scatt_molden_close.argtypes = [vp]
    _bound = True


def read_molden(path) -> dict:
    """atoms (n, 4: Z, x, y, z bohr), shells [(centre, l, exponents, raw
    coefficients)], nbf, and per spin ('alpha', 'beta') the MO coefficients
    (n_mo, nbf), occupations and energies.  Raises ScattError on a malformed
    file or a Cartesian shell of l >= 2."""
    _bind()
    L = lib()
    h = C.c_void_p()
    check(L.scatt_molden_open(os.fsencode(os.fspath(path)), C.byref(h)))
    try:
        info = np.zeros(7, dtype=np.int32)
        check(L.scatt_molden_info(h, as_iptr(info)))
        n_atoms, n_shell, nbf, n_a, n_b, n_prim, _ = (int(x) for x in info)
        atoms = np.zeros((n_atoms, 4))
        check(L.scatt_molden_atoms(h, as_dptr(atoms)))
        l = np.zeros(n_shell, dtype=np.int32)
        npr = np.zeros(n_shell, dtype=np.int32)
        cen = np.zeros((n_shell, 3))
        ex = np.zeros(max(n_prim, 1))
        cf = np.zeros(max(n_prim, 1))
        check(L.scatt_molden_shells(h, as_iptr(l), as_iptr(npr), as_dptr(cen), as_dptr(ex), as_dptr(cf)))
        shells, p = [], 0
        for i in range(n_shell):
            shells.append((cen[i].copy(), int(l[i]), ex[p:p + npr[i]].copy(), cf[p:p + npr[i]].copy()))
            p += int(npr[i])
        out = {"atoms": atoms, "shells": shells, "nbf": nbf}
        for spin, n in (("alpha", n_a), ("beta", n_b)):
            Cm, occ, ene = np.zeros((n, nbf)), np.zeros(n), np.zeros(n)
            if n:
                check(L.scatt_molden_mos(h, 1 if spin == "beta" else 0, as_dptr(Cm), as_dptr(occ), as_dptr(ene)))
            out[spin] = {"C": Cm, "occ": occ, "energy": ene}
        return out
    finally:
        L.scatt_molden_close(h)

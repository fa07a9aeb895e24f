"""Host-side interface of the per-energy scattering solver (ctypes over the C ABI).

``ScanSolver`` mirrors the reference's run_one_energy pipeline
(src/main.cpp:1081-1623) for a batch of energies: the scan's static inputs are
uploaded once (scatt_upload_static), then any number of energies are solved
(scatt_solve_batch).  Results come back as numpy arrays named after the
reference's result structs (ScatteringResult, AmplitudeResult,
DipoleResult).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import as_dptr, check, dptr, iptr, lib

SLOTS = [("length", "x"), ("length", "y"), ("length", "z"),
         ("velocity", "x"), ("velocity", "y"), ("velocity", "z")]

DIAG = ["fit_residual_max", "fit_residual_rel", "A_minus_I_max", "K_symmetry_err_aa",
        "S_unitarity_err_aa", "K_symmetry_err_kme", "unitarity_err_kme", "n_fit_start",
        "n_fit_end", "n_transition", "shifts_A", "shifts_S", "n_closed_l", "schur_coupling_zero"]
NDIAG = 16


class ScanDesc(C.Structure):
    _fields_ = [("Nr", C.c_int), ("dr", C.c_double), ("l_cont_max", C.c_int), ("n_occ", C.c_int),
                ("n_orb", C.c_int), ("Nlm_store", C.c_int), ("Nr_store", C.c_int), ("psi_lm", dptr),
                ("init_state", C.c_int), ("n_H", C.c_int), ("V_H", dptr), ("n_atoms", C.c_int),
                ("atoms", dptr), ("alpha_pol", C.c_double), ("pol_form", C.c_int), ("r_c", C.c_double),
                ("n_transition", C.c_int), ("chi_cutoff", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("W_min", C.c_double), ("stab_n_max", C.c_int), ("shift_margin", C.c_double),
                ("n_asym", C.c_int), ("allow_closed_channels", C.c_int), ("orthogonalize", C.c_int),
                ("max_batch", C.c_int), ("use_graphs", C.c_int), ("diagnostics", C.c_int),
                ("timing", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [(n, dptr) for n in ("K_kme", "A", "B", "K_aa", "b_overlap", "D_re", "D_im", "Draw_re",
                                    "Draw_im", "d_raw", "d_corr", "partial_sigma", "eig_kme", "eig_aa",
                                    "diag")] + [("status", iptr)]


_bound = False


def _bind():
    global _bound
    if _bound:
        return
    L = lib()
    L.scatt_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    L.scatt_ctx_destroy.argtypes = [C.c_void_p]
    L.scatt_upload_static.argtypes = [C.c_void_p, C.POINTER(ScanDesc)]
    L.scatt_scan_info.argtypes = [C.c_void_p, iptr]
    L.scatt_solve_batch.argtypes = [C.c_void_p, C.c_int, dptr, iptr, C.POINTER(SolveOpts), C.POINTER(Outputs)]
    L.scatt_default_opts.argtypes = [C.POINTER(SolveOpts)]
    L.scatt_default_opts.restype = None
    L.scatt_last_stats.argtypes = [C.c_void_p, dptr]
    _bound = True


def default_opts(**kw) -> SolveOpts:
    _bind()
    o = SolveOpts()
    lib().scatt_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


@dataclass
class EnergyResult:
    """Per-energy outputs (views into the batch arrays)."""
    E: float
    K_kme: np.ndarray
    A: np.ndarray
    B: np.ndarray
    K_aa: np.ndarray
    b_overlap: np.ndarray
    D: np.ndarray            # (6, Np) complex, D_reduced
    D_raw: np.ndarray        # (6, Np) complex, D_reduced_raw
    d_raw: np.ndarray        # (6, Np)
    d_corr: np.ndarray       # (6, n_occ)
    partial_sigma: np.ndarray  # (6,)
    eig_kme: np.ndarray
    eig_aa: np.ndarray
    diag: dict
    status: int


class ScanSolver:
    """One scan (static inputs resident on the device) solving batches of energies."""

    def __init__(self, inp, device: int = 0, l_cont_max: int | None = None, n_transition: int = 0):
        _bind()
        self._ctx = C.c_void_p()
        check(lib().scatt_ctx_create(device, C.byref(self._ctx)))
        self.inp = inp
        self.l_cont_max = inp.l_cont if l_cont_max is None else l_cont_max
        self._keep = []
        psi = np.ascontiguousarray(inp.psi_lm, dtype=np.float64)
        vh = np.ascontiguousarray(inp.V_H, dtype=np.float64)
        at = np.ascontiguousarray(inp.atoms, dtype=np.float64)
        self._keep += [psi, vh, at]
        d = ScanDesc()
        d.Nr, d.dr, d.l_cont_max = inp.Nr, inp.dr, self.l_cont_max
        d.n_occ = inp.n_occ
        d.n_orb, d.Nlm_store, d.Nr_store = psi.shape
        d.psi_lm = as_dptr(psi)
        d.init_state = inp.init_state
        d.n_H = vh.shape[0]
        d.V_H = as_dptr(vh)
        d.n_atoms = at.shape[0]
        d.atoms = as_dptr(at)
        d.alpha_pol, d.pol_form, d.r_c = inp.alpha_pol, inp.pol_form, inp.r_c
        d.n_transition = n_transition
        d.chi_cutoff = 1e-15
        check(lib().scatt_upload_static(self._ctx, C.byref(d)))
        info = np.zeros(5, dtype=np.int32)
        check(lib().scatt_scan_info(self._ctx, info.ctypes.data_as(iptr)))
        self.n_transition, self.Np, self.Nf, self.n_lambda, self.n_sigma = (int(x) for x in info)
        self.n_occ = inp.n_occ

    def close(self):
        if self._ctx:
            lib().scatt_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_stats(self) -> dict:
        """Device timing of the last solve (needs opts.timing = 1)."""
        v = np.zeros(6)
        check(lib().scatt_last_stats(self._ctx, as_dptr(v)))
        return {"device_s": v[0], "rinv_s": v[1], "rinv_calls": int(v[2]), "launches": int(v[3]),
                "sweep_s": v[4], "post_s": v[5]}

    def solve(self, energies, l_cont=None, opts: SolveOpts | None = None, raise_on_error=True):
        E = np.ascontiguousarray(energies, dtype=np.float64).reshape(-1)
        nE = E.size
        Np, no = self.Np, self.n_occ
        lc = None
        if l_cont is not None:
            lc = np.ascontiguousarray(np.broadcast_to(np.asarray(l_cont, dtype=np.int32), (nE,)))
        arr = {
            "K_kme": np.zeros((nE, Np, Np)), "A": np.zeros((nE, Np, Np)), "B": np.zeros((nE, Np, Np)),
            "K_aa": np.zeros((nE, Np, Np)), "b_overlap": np.zeros((nE, no, Np)),
            "D_re": np.zeros((nE, 6, Np)), "D_im": np.zeros((nE, 6, Np)), "Draw_re": np.zeros((nE, 6, Np)),
            "Draw_im": np.zeros((nE, 6, Np)), "d_raw": np.zeros((nE, 6, Np)), "d_corr": np.zeros((nE, 6, no)),
            "partial_sigma": np.zeros((nE, 6)), "eig_kme": np.zeros((nE, Np)), "eig_aa": np.zeros((nE, Np)),
            "diag": np.zeros((nE, NDIAG)),
        }
        status = np.zeros(nE, dtype=np.int32)
        out = Outputs()
        for k, v in arr.items():
            setattr(out, k, as_dptr(v))
        out.status = status.ctypes.data_as(iptr)
        o = opts if opts is not None else default_opts()
        code = lib().scatt_solve_batch(self._ctx, nE, as_dptr(E),
                                       lc.ctypes.data_as(iptr) if lc is not None else None,
                                       C.byref(o), C.byref(out))
        if code != 0 and raise_on_error:
            check(code)
        res = []
        for e in range(nE):
            n = (int(lc[e]) + 1) ** 2 if lc is not None else Np
            # matrices come back column-major: transpose the C-order view
            mat = lambda a: a[e].T[:n, :n]
            res.append(EnergyResult(
                E=float(E[e]), K_kme=mat(arr["K_kme"]), A=mat(arr["A"]), B=mat(arr["B"]),
                K_aa=mat(arr["K_aa"]), b_overlap=arr["b_overlap"][e].T[:n, :],
                D=(arr["D_re"][e] + 1j * arr["D_im"][e])[:, :n],
                D_raw=(arr["Draw_re"][e] + 1j * arr["Draw_im"][e])[:, :n],
                d_raw=arr["d_raw"][e][:, :n], d_corr=arr["d_corr"][e], partial_sigma=arr["partial_sigma"][e],
                eig_kme=arr["eig_kme"][e][:n], eig_aa=arr["eig_aa"][e][:n],
                diag={k: arr["diag"][e][i] for i, k in enumerate(DIAG)}, status=int(status[e])))
        return res

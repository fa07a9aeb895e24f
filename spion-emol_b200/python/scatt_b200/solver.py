"""Host-side interface of the per-energy scattering solver (ctypes over the C ABI).

``ScanSolver`` mirrors the reference's run_one_energy pipeline
(src/main.cpp:1081-1623) for a batch of energies: the scan's static inputs are
uploaded once (scatt_upload_static), then any number of energies are solved
(scatt_solve_batch).  Results come back as numpy arrays named after the
reference's result structs (ScatteringResult, AmplitudeResult,
DipoleResult).

``Scan`` (ScanSolver.scan) is the streaming form of the same solve: energies
are queued, run in phase-staggered slot groups, and come back as each group
finishes (scatt_scan_open / submit / step / close).
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
                ("timing", C.c_int), ("keep_window", C.c_int)]


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
    L.scatt_scan_open.argtypes = [C.c_void_p, C.POINTER(SolveOpts), C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_void_p)]
    L.scatt_scan_submit.argtypes = [C.c_void_p, C.c_int, dptr, iptr]
    L.scatt_scan_step.argtypes = [C.c_void_p, C.POINTER(Outputs), C.c_int, iptr, C.POINTER(C.c_longlong)]
    L.scatt_scan_pending.argtypes = [C.c_void_p, iptr, iptr]
    L.scatt_scan_shape.argtypes = [C.c_void_p, iptr, iptr]
    L.scatt_scan_close.argtypes = [C.c_void_p]
    L.scatt_psi_sweep.argtypes = [C.c_void_p, C.POINTER(SolveOpts), C.c_int, dptr, iptr, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(Outputs), dptr]
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
        self.dr = float(inp.dr)
        self.device = int(device)
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
        self._upload(d)

    @classmethod
    def from_preproc(cls, path, l_cont_max: int, device: int = 0, n_transition: int = 0) -> "ScanSolver":
        """A solver on a preprocessing file in the reference's schema (split
        or combined layout; see h5io.Preproc).  self.E_init is the dipole
        initial state's energy, self.preproc the opened file's header."""
        from .h5io import Preproc
        _bind()
        self = cls.__new__(cls)
        self._ctx = C.c_void_p()
        check(lib().scatt_ctx_create(device, C.byref(self._ctx)))
        self.inp = None
        self.device = int(device)
        self.l_cont_max = int(l_cont_max)
        self._keep = []
        with Preproc(path) as pp:
            d, self.E_init = pp.desc(l_cont_max)
            self.dr = float(pp.dr)
            d.n_transition = n_transition
            self._upload(d)                  # copies to the device before the file's buffers go
            self.preproc = {k: getattr(pp, k) for k in ("Nr", "dr", "Lmax_sce", "n_alpha", "n_occ", "n_sce",
                                                        "Nlm_orb_store", "Nr_orb_store", "has_initial_state")}
            self.orb_energies = pp.orb_energies.copy()
            self.atoms = pp.atoms.copy()
        return self

    def _upload(self, d):
        check(lib().scatt_upload_static(self._ctx, C.byref(d)))
        info = np.zeros(5, dtype=np.int32)
        check(lib().scatt_scan_info(self._ctx, info.ctypes.data_as(iptr)))
        self.n_transition, self.Np, self.Nf, self.n_lambda, self.n_sigma = (int(x) for x in info)
        self.n_occ = d.n_occ

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
        """Device timing of the last solve, or of the open scan's steps so far
        (needs opts.timing = 1)."""
        v = np.zeros(7)
        check(lib().scatt_last_stats(self._ctx, as_dptr(v)))
        return {"device_s": v[0], "rinv_s": v[1], "rinv_calls": int(v[2]), "launches": int(v[3]),
                "sweep_s": v[4], "post_s": v[5], "rinv_flops": v[6]}

    def solve(self, energies, l_cont=None, opts: SolveOpts | None = None, raise_on_error=True):
        E = np.ascontiguousarray(energies, dtype=np.float64).reshape(-1)
        nE = E.size
        lc = None
        if l_cont is not None:
            lc = np.ascontiguousarray(np.broadcast_to(np.asarray(l_cont, dtype=np.int32), (nE,)))
        arr, status, out = output_arrays(nE, self.Np, self.n_occ)
        o = opts if opts is not None else default_opts()
        code = lib().scatt_solve_batch(self._ctx, nE, as_dptr(E),
                                       lc.ctypes.data_as(iptr) if lc is not None else None,
                                       C.byref(o), C.byref(out))
        if code != 0 and raise_on_error:
            check(code)
        return [result_of(arr, status, e, float(E[e]), int(lc[e]) if lc is not None else None, self.Np)
                for e in range(nE)]

    def psi_sweep(self, energies, n_lo: int = 0, n_hi: int | None = None, segment: int = 64, l_cont=None,
                  opts: SolveOpts | None = None, alloc=None, raise_on_error=True):
        """psi(n) for n_lo <= n < n_hi (default: the whole grid) of every
        energy, by the back-propagation of BackPropagator::run / get_psi
        (scatt_psi_sweep), with the energies' results.

        Returns (results, psi): psi[i, r] is psi(n_lo + r) of energy i as an
        Np_max x Np_max array, rows = channel, columns = solution (zero
        outside the energy's own block).  alloc(shape, dtype) may supply the
        host buffer -- page-locked memory lets the device-to-host copies
        overlap the sweep."""
        E = np.ascontiguousarray(energies, dtype=np.float64).reshape(-1)
        nE = E.size
        n_hi = self.inp.Nr if n_hi is None and self.inp is not None else n_hi
        if n_hi is None:
            n_hi = int(self.preproc["Nr"])
        lc = None
        if l_cont is not None:
            lc = np.ascontiguousarray(np.broadcast_to(np.asarray(l_cont, dtype=np.int32), (nE,)))
        arr, status, out = output_arrays(nE, self.Np, self.n_occ)
        mk = alloc or (lambda shape, dtype=np.float64: np.zeros(shape, dtype=dtype))
        buf = mk((nE, n_hi - n_lo, self.Np, self.Np))
        o = opts if opts is not None else default_opts()
        code = lib().scatt_psi_sweep(self._ctx, C.byref(o), nE, as_dptr(E),
                                     lc.ctypes.data_as(iptr) if lc is not None else None,
                                     int(segment), int(n_lo), int(n_hi), C.byref(out), as_dptr(buf))
        if code != 0 and raise_on_error:
            check(code)
        res = [result_of(arr, status, e, float(E[e]), int(lc[e]) if lc is not None else None, self.Np)
               for e in range(nE)]
        # column-major matrices: the transposed view of each C-order slab
        return res, np.swapaxes(buf, 2, 3)

    def scan(self, slots: int = 0, groups: int = 1, l_cont_max: int | None = None,
             opts: SolveOpts | None = None, alloc=None) -> "Scan":
        """A streaming scan over this solver's static inputs (see Scan)."""
        return Scan(self, slots, groups, l_cont_max, opts, alloc)


def output_arrays(nE, Np, no, alloc=None):
    """Host output arrays for nE energies and the scatt_outputs pointing at
    them; alloc(shape, dtype) may supply the memory (e.g. pinned)."""
    mk = alloc or (lambda shape, dtype=np.float64: np.zeros(shape, dtype=dtype))
    arr = {
        "K_kme": mk((nE, Np, Np)), "A": mk((nE, Np, Np)), "B": mk((nE, Np, Np)),
        "K_aa": mk((nE, Np, Np)), "b_overlap": mk((nE, no, Np)),
        "D_re": mk((nE, 6, Np)), "D_im": mk((nE, 6, Np)), "Draw_re": mk((nE, 6, Np)),
        "Draw_im": mk((nE, 6, Np)), "d_raw": mk((nE, 6, Np)), "d_corr": mk((nE, 6, no)),
        "partial_sigma": mk((nE, 6)), "eig_kme": mk((nE, Np)), "eig_aa": mk((nE, Np)),
        "diag": mk((nE, NDIAG)),
    }
    status = mk((nE,), np.int32)
    out = Outputs()
    for k, v in arr.items():
        setattr(out, k, as_dptr(v))
    out.status = status.ctypes.data_as(iptr)
    return arr, status, out


def output_bytes(arr, status, rows: int) -> int:
    """Bytes of `rows` energies' outputs (what a device-to-host read moves)."""
    return int(sum(v[:rows].nbytes for v in arr.values()) + status[:rows].nbytes)


def result_of(arr, status, e, E, l_cont, Np) -> EnergyResult:
    n = (l_cont + 1) ** 2 if l_cont is not None else Np
    # matrices come back column-major: transpose the C-order view (copies, so
    # a result outlives the buffer's next use)
    mat = lambda a: np.array(a[e].T[:n, :n])
    return EnergyResult(
        E=E, K_kme=mat(arr["K_kme"]), A=mat(arr["A"]), B=mat(arr["B"]),
        K_aa=mat(arr["K_aa"]), b_overlap=np.array(arr["b_overlap"][e].T[:n, :]),
        D=(arr["D_re"][e] + 1j * arr["D_im"][e])[:, :n],
        D_raw=(arr["Draw_re"][e] + 1j * arr["Draw_im"][e])[:, :n],
        d_raw=np.array(arr["d_raw"][e][:, :n]), d_corr=np.array(arr["d_corr"][e]),
        partial_sigma=np.array(arr["partial_sigma"][e]),
        eig_kme=np.array(arr["eig_kme"][e][:n]), eig_aa=np.array(arr["eig_aa"][e][:n]),
        diag={k: float(arr["diag"][e][i]) for i, k in enumerate(DIAG)}, status=int(status[e]))


class Scan:
    """Streaming scan (scatt_scan_*): energies wait in a queue and run in
    `slots` device slots split into `groups` phase groups.  The groups start
    staggered by a fraction of the radial sweep, so once the conveyor is full
    a group finishes every 1/groups of a sweep and its slots take the next
    queued energies; every slot stays busy while the queue lasts.
    groups = 1 is the lock-step batch of ScanSolver.solve."""

    def __init__(self, solver: ScanSolver, slots=0, groups=1, l_cont_max=None, opts=None, alloc=None):
        _bind()
        self.solver = solver
        self._h = C.c_void_p()
        self.l_cont_max = solver.l_cont_max if l_cont_max is None else l_cont_max
        o = opts if opts is not None else default_opts()
        check(lib().scatt_scan_open(solver._ctx, C.byref(o), int(slots), int(groups), int(self.l_cont_max),
                                    C.byref(self._h)))
        sl, gr = C.c_int(0), C.c_int(0)
        check(lib().scatt_scan_shape(self._h, C.byref(sl), C.byref(gr)))
        self.slots, self.groups = sl.value, gr.value
        self.arr, self.status, self._out = output_arrays(self.slots, solver.Np, solver.n_occ, alloc)
        self._idx = np.zeros(self.slots, dtype=np.int64)
        self._E, self._lc = [], []
        self.last_out_bytes = 0

    def submit(self, energies, l_cont=None):
        """Queue energies; returns their submission indices."""
        E = np.ascontiguousarray(energies, dtype=np.float64).reshape(-1)
        lc = None
        if l_cont is not None:
            lc = np.ascontiguousarray(np.broadcast_to(np.asarray(l_cont, dtype=np.int32), (E.size,)))
        check(lib().scatt_scan_submit(self._h, E.size, as_dptr(E),
                                      lc.ctypes.data_as(iptr) if lc is not None else None))
        first = len(self._E)
        self._E += [float(x) for x in E]
        self._lc += [int(x) for x in lc] if lc is not None else [None] * E.size
        return list(range(first, first + E.size))

    def step(self, raise_on_error=True, results=True):
        """Advance until the next group finishes; [(submission index, EnergyResult)]
        (an empty list once nothing is queued or in flight).  results=False
        returns the indices only and leaves the outputs in self.arr."""
        n = C.c_int(0)
        code = lib().scatt_scan_step(self._h, C.byref(self._out), self.slots, C.byref(n),
                                     self._idx.ctypes.data_as(C.POINTER(C.c_longlong)))
        if code != 0 and raise_on_error:
            check(code)
        self.last_out_bytes = output_bytes(self.arr, self.status, n.value)
        idx = [int(self._idx[i]) for i in range(n.value)]
        if not results:
            return idx
        return [(j, result_of(self.arr, self.status, i, self._E[j], self._lc[j], self.solver.Np))
                for i, j in enumerate(idx)]

    def pending(self):
        q, f = C.c_int(0), C.c_int(0)
        check(lib().scatt_scan_pending(self._h, C.byref(q), C.byref(f)))
        return q.value, f.value

    def close(self):
        if self._h:
            lib().scatt_scan_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

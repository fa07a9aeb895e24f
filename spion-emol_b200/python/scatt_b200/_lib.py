"""ctypes binding of libscatt_b200.so (the C ABI declared in include/scatt_b200.h).

The library is built in-tree (spion-emol_b200/libscatt_b200.so).  Loading it
does not need a GPU; every compute entry point returns SCATT_ERR_NO_DEVICE
when none is visible, and this module turns non-zero statuses into
ScattError.  There is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(os.path.dirname(_HERE))          # spion-emol_b200/
LIB_PATH = os.path.join(PKG_ROOT, "libscatt_b200.so")

STATUS = {
    0: "SCATT_OK", 1: "SCATT_ERR_ARG", 2: "SCATT_ERR_CUDA", 3: "SCATT_ERR_SIZE",
    4: "SCATT_ERR_SINGULAR", 5: "SCATT_ERR_NONFINITE", 6: "SCATT_ERR_CLOSED_CHANNEL",
    7: "SCATT_ERR_NO_DEVICE", 8: "SCATT_ERR_STATE", 9: "SCATT_ERR_OOM", 10: "SCATT_ERR_FIT_WINDOW",
    11: "SCATT_ERR_IO",
}


class ScattError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


_lib = None

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int)


def lib():
    """Load (once) and return the CDLL with argtypes set."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ScattError(2, f"{LIB_PATH} is missing: build it with python spion-emol_b200/build.py")
    L = C.CDLL(LIB_PATH)
    L.scatt_version.restype = C.c_char_p
    L.scatt_last_error.restype = C.c_char_p
    L.scatt_device_count.argtypes = [iptr]
    for f in ("scatt_wigner3j", "scatt_gaunt_real"):
        getattr(L, f).restype = C.c_double
        getattr(L, f).argtypes = [C.c_int] * 6
    L.scatt_angular_dipole.restype = C.c_double
    L.scatt_angular_dipole.argtypes = [C.c_int] * 5
    L.scatt_velocity_coef.restype = C.c_double
    L.scatt_velocity_coef.argtypes = [C.c_int] * 2
    for f in ("scatt_riccati_j", "scatt_riccati_y"):
        getattr(L, f).restype = C.c_double
        getattr(L, f).argtypes = [C.c_int, C.c_double]
    L.scatt_inverse_batched.argtypes = [C.c_int, C.c_int, dptr, dptr, C.c_int, iptr]
    L.scatt_inverse_batched_noalloc.argtypes = [C.c_int, C.c_int, dptr, dptr, C.c_int, iptr]
    L.scatt_dgemm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                              dptr, C.c_int, dptr, C.c_int, C.c_double, dptr, C.c_int]
    L.scatt_bench_inverse.argtypes = [C.c_int, C.c_int, C.c_int, dptr]
    L.scatt_bench_gemm.argtypes = [C.c_int] * 8 + [dptr]
    L.scatt_set_inverse_blocking.argtypes = [C.c_int]
    L.scatt_sce_grid.argtypes = [C.c_int, dptr, dptr, dptr]
    L.scatt_sce_project.argtypes = [C.c_int, C.c_int, C.c_int, dptr, dptr]
    L.scatt_sce_basis.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, dptr, C.c_int, iptr, iptr, dptr, dptr,
                                  dptr, C.c_int, dptr, dptr, C.c_int, C.c_int, dptr, dptr, dptr]
    L.scatt_hartree.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, dptr, dptr]
    L.scatt_cc_dipole.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, dptr, C.c_int, dptr, dptr]
    _lib = L
    return L


def check(code: int):
    if code != 0:
        raise ScattError(code, lib().scatt_last_error().decode())


def as_dptr(a: np.ndarray):
    return a.ctypes.data_as(dptr)


def as_iptr(a: np.ndarray):
    return a.ctypes.data_as(iptr)


def device_count() -> int:
    n = C.c_int(0)
    check(lib().scatt_device_count(C.byref(n)))
    return n.value


def inverse_batched(A: np.ndarray, symmetrize: bool = False, noalloc: bool = False):
    """Inverse of each n x n matrix of A (shape (count, n, n) or (n, n)); returns (inv, status).

    noalloc=True goes through scatt_inverse_batched_noalloc (static device
    scratch, no device allocation; bounded sizes)."""
    A = np.asarray(A, dtype=np.float64)
    single = A.ndim == 2
    if single:
        A = A[None]
    count, n, _ = A.shape
    # column-major per matrix: pass the transpose's memory
    Af = np.ascontiguousarray(np.transpose(A, (0, 2, 1)))
    out = np.empty_like(Af)
    st = np.zeros((count, 2), dtype=np.int32)
    fn = lib().scatt_inverse_batched_noalloc if noalloc else lib().scatt_inverse_batched
    code = fn(n, count, as_dptr(Af), as_dptr(out), int(symmetrize), as_iptr(st))
    inv = np.transpose(out, (0, 2, 1))
    if code not in (0, 4, 5):
        check(code)
    return (inv[0] if single else inv), st


def dgemm(A, B, C=None, alpha=1.0, beta=0.0, opA=0, opB=0):
    """alpha op(A) op(B) + beta C on the device."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    M = A.shape[1] if opA else A.shape[0]
    K = A.shape[0] if opA else A.shape[1]
    N = B.shape[0] if opB else B.shape[1]
    Cm = np.zeros((M, N), order="F") if C is None else np.array(C, dtype=np.float64, order="F", copy=True)
    check(lib().scatt_dgemm(opA, opB, M, N, K, alpha, as_dptr(A), A.shape[0], as_dptr(B), B.shape[0],
                            beta, as_dptr(Cm), M))
    return Cm


def bench_inverse(n: int, count: int, reps: int = 5) -> float:
    ms = C.c_double(0.0)
    check(lib().scatt_bench_inverse(n, count, reps, C.byref(ms)))
    return ms.value


def bench_gemm(opA: int, opB: int, M: int, N: int, K: int, count: int, sym: bool = False, reps: int = 5) -> float:
    """Milliseconds of one batched GEMM call on device-resident operands (scatt_bench_gemm)."""
    ms = C.c_double(0.0)
    check(lib().scatt_bench_gemm(int(opA), int(opB), int(M), int(N), int(K), int(count), 1 if sym else 0,
                                 int(reps), C.byref(ms)))
    return ms.value


def autotune_inverse(n: int, count: int, reps: int = 3, device: int | None = None) -> dict:
    """Time the two-level inverse's configurations for order n and batch
    `count` on the current (or given) device and keep the fastest for every
    later inverse of that order and batch (scatt_autotune_inverse)."""
    if device is not None:
        import torch
        torch.cuda.set_device(device)
    sc, pc, la, win = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
    ms = C.c_double(0.0)
    check(lib().scatt_autotune_inverse(int(n), int(count), int(reps), C.byref(sc), C.byref(pc), C.byref(la),
                                       C.byref(win), C.byref(ms)))
    return {"n": int(n), "count": int(count), "scheme": sc.value, "panel": pc.value,
            "look_ahead": la.value, "window": win.value, "ms": ms.value}


def set_inverse_blocking(scheme: int):
    """0: automatic (default); 1: single-level; 2: two-level column-major;
    3: two-level row-contiguous; 4: as 3 with 128-column windows; 5, 6: as 3, 4
    with the small cluster panel."""
    check(lib().scatt_set_inverse_blocking(int(scheme)))


CC_Q = {"x": 1, "y": -1, "z": 0}       # CCDipole.cpp: q of each polarisation


def cc_dipole(psi_kappa, psi_nu, ir0: int, dr: float, pol: str, n_mu: int | None = None) -> np.ndarray:
    """Continuum-continuum dipoles of one final state against n_nu
    intermediate states on the device (scatt_cc_dipole), length gauge.

    psi_kappa: (n_pts, L, L) with psi_kappa[i] = psi(ir0 + i) (rows =
    channel, columns = solution; one energy of ScanSolver.psi_sweep's
    output); psi_nu: (n_nu, n_pts, L, L) or (n_pts, L, L).  n_mu (default
    L): the leading block used.  Returns (n_nu, n_mu, n_mu) with
    cc[v][beta, alpha] = sum_i w_i r_i psi_kappa(i)[:, beta] . A^q psi_nu_v(i)[:, alpha]."""
    pk = np.asarray(psi_kappa, dtype=np.float64)
    pn = np.asarray(psi_nu, dtype=np.float64)
    if pn.ndim == 3:
        pn = pn[None]
    n_pts, L = pk.shape[0], pk.shape[1]
    if pn.shape[1:] != pk.shape:
        raise ValueError("psi_nu stacks must match psi_kappa's shape")
    n_mu = L if n_mu is None else int(n_mu)
    # column-major matrices: the C-order buffers of the transposed views
    ck = np.ascontiguousarray(np.swapaxes(pk, -1, -2))
    cn = np.ascontiguousarray(np.swapaxes(pn, -1, -2))
    out = np.zeros((pn.shape[0], n_mu, n_mu))
    check(lib().scatt_cc_dipole(n_mu, L, n_pts, int(ir0), float(dr), CC_Q[pol], as_dptr(ck), pn.shape[0],
                                as_dptr(cn), as_dptr(out)))
    return np.swapaxes(out, 1, 2)


def hartree(rho_lm, dr: float, l_max: int, r0: float = 0.0) -> np.ndarray:
    """V_H multipoles ((l_max + 1)^2, Nr) from the density multipoles rho_lm
    (>= (l_max + 1)^2 rows, Nr columns) by the radial Poisson integrals of
    the preprocessing step, on the device (scatt_hartree)."""
    rho = np.ascontiguousarray(rho_lm, dtype=np.float64)
    n_lm = (int(l_max) + 1) ** 2
    out = np.zeros((n_lm, rho.shape[1]))
    check(lib().scatt_hartree(int(l_max), rho.shape[0], rho.shape[1], float(r0), float(dr), as_dptr(rho),
                              as_dptr(out)))
    return out


def sce_grid(Lmax: int):
    """(cos_theta, weights, phi) of the single-centre expansion's angular grid."""
    x, w, p = np.zeros(Lmax + 1), np.zeros(Lmax + 1), np.zeros(2 * (Lmax + 1))
    check(lib().scatt_sce_grid(int(Lmax), as_dptr(x), as_dptr(w), as_dptr(p)))
    return x, w, p


def sce_project(samples, Lmax: int, chunk: int = 0) -> np.ndarray:
    """F_lm ((Lmax + 1)^2, Nr) from samples (Nr, n_theta, n_phi) of F on the
    grid of sce_grid(Lmax), on the device (scatt_sce_project)."""
    X = np.ascontiguousarray(samples, dtype=np.float64)
    Nr = X.shape[0]
    if X.shape[1:] != (Lmax + 1, 2 * (Lmax + 1)):
        raise ValueError("samples must be (Nr, Lmax + 1, 2 (Lmax + 1))")
    out = np.zeros(((Lmax + 1) ** 2, Nr))
    check(lib().scatt_sce_project(int(Lmax), Nr, int(chunk), as_dptr(X), as_dptr(out)))
    return out


def sce_basis(shells, C_mo, occ, Lmax: int, Nr: int, r0: float, dr: float, origin=(0.0, 0.0, 0.0),
              chunk: int = 0, vx_form: int = 0):
    """(orb_lm (n_mo, Nlm, Nr), rho_lm (Nlm, Nr)), and vx_lm (Nlm, Nr) when
    vx_form is 1 (Slater) or 2 (Kohn-Sham): the single-centre expansions of
    the molecular orbitals, the density and the local exchange of a
    contracted spherical-Gaussian basis on the device (scatt_sce_basis).
    shells: a list of (center (3,), l, exponents, raw coefficients); C_mo:
    (n_mo, nbf) in molden AO order; occ: (n_mo,)."""
    sl = np.array([int(s[1]) for s in shells], dtype=np.int32)
    sn = np.array([len(s[2]) for s in shells], dtype=np.int32)
    sc = np.ascontiguousarray([np.asarray(s[0], dtype=np.float64) for s in shells])
    ex = np.ascontiguousarray(np.concatenate([np.asarray(s[2], dtype=np.float64) for s in shells]))
    cf = np.ascontiguousarray(np.concatenate([np.asarray(s[3], dtype=np.float64) for s in shells]))
    Cm = np.ascontiguousarray(C_mo, dtype=np.float64)
    oc = np.ascontiguousarray(occ, dtype=np.float64)
    o = np.ascontiguousarray(origin, dtype=np.float64)
    n_lm = (Lmax + 1) ** 2
    orb = np.zeros((Cm.shape[0], n_lm, Nr))
    rho = np.zeros((n_lm, Nr))
    vx = np.zeros((n_lm, Nr)) if vx_form else None
    check(lib().scatt_sce_basis(int(Lmax), int(Nr), float(r0), float(dr), as_dptr(o), len(shells), as_iptr(sl),
                                as_iptr(sn), as_dptr(sc), as_dptr(ex), as_dptr(cf), Cm.shape[0], as_dptr(Cm),
                                as_dptr(oc), int(vx_form), int(chunk), as_dptr(orb), as_dptr(rho),
                                as_dptr(vx) if vx is not None else None))
    return (orb, rho, vx) if vx_form else (orb, rho)

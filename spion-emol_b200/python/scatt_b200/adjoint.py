"""Gradients of dipoles, cross sections and time delays (device adjoint).

The reference has no adjoint.  Here the forward recurrence, its checkpoints
and the reverse pass run in libscatt_b200 (scatt_adjoint_*); the small
stages after the radial sweep -- K extraction (KMatrixExtractor.cpp:75-198),
the outer boundary and the fit-window back sweep (BackPropagator.cpp:127-197,
603-703), the fit (AsymptoticAmplitudes.cpp:64-359) and the dipole algebra
(DipoleMatrixElement.cpp:673-947) -- run in torch on the GPU, on zero-copy
views of the library's window store, so autograd differentiates them.  Their
cotangents (dJ/dRinv and dJ/dSinv over the window, dJ/dG(N-1)) go back to
the library, whose reverse pass returns tr dJ/dV(n) per energy and,
optionally, dJ/dV(n) summed over the energies.

    D = Dipoles.apply(alpha, r_c, dV, solver, energies)   # (n_energy, 6, Np, 2)
    obs = observables(energies, D, e_homo)                  # sigma_*, tau_*
    obs["sigma_length_z"].sum().backward()                  # -> alpha.grad, r_c.grad, dV.grad

V_pol = -alpha / (2 (r^2 + r_c^2)^2) (form 1) or the reference's damped form
(form 0, Potentials.cpp:111-129) enters V(n) on the diagonal; its parameter
gradients are sum_n tr(dJ/dV(n)) dV_pol(r_n)/dparam.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import solver as S
from ._lib import ScattError, as_dptr, check, lib

F64 = torch.float64
C_AU = 137.036


class AdjView(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("N", "n_s", "n_window", "n_tr", "n_pts", "n_start", "ne_fit", "Np", "Nt",
                                        "Nf", "Krows", "Np_max", "l_cont")] + \
               [("E", C.c_double)] + \
               [(n, C.c_void_p) for n in ("Rwin", "Swin", "G_last", "RBwin", "SBwin", "GB_last", "V_N", "B_N",
                                          "Bs_N", "C_N", "Bs_win")]


_bound = False


def _bind():
    global _bound
    if _bound:
        return
    S._bind()
    L = lib()
    vp = C.c_void_p
    L.scatt_set_polarization.argtypes = [vp, C.c_double, C.c_double, C.c_int]
    L.scatt_set_potential_delta.argtypes = [vp, vp]
    L.scatt_adjoint_forward.argtypes = [vp, C.POINTER(S.SolveOpts), C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_int), C.c_int, C.POINTER(S.Outputs), C.POINTER(vp)]
    L.scatt_adjoint_view_of.argtypes = [vp, C.c_int, C.POINTER(AdjView)]
    L.scatt_adjoint_reverse.argtypes = [vp, C.POINTER(C.c_double), vp]
    L.scatt_adjoint_close.argtypes = [vp]
    L.scatt_riccati_j.restype = C.c_double
    L.scatt_riccati_y.restype = C.c_double
    _bound = True


class _Dev:
    """A device array handed to torch without a copy (CUDA array interface)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(int(x) for x in shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def _raw(ptr, shape, device):
    """Row-major torch view of `shape` over device memory at ptr (a column-major
    n x m matrix is the raw (m, n) view, i.e. its transpose)."""
    if not ptr:
        return None
    return torch.as_tensor(_Dev(ptr, shape), device=device)


def _rj(l, x):
    return lib().scatt_riccati_j(int(l), float(x))


def _ry(l, x):
    return lib().scatt_riccati_y(int(l), float(x))


def _sym(M):
    return 0.5 * (M + M.transpose(-1, -2))


def vpol(r, alpha, r_c, pol_form: int):
    """V_pol on radii r (tensor), as the device's k_build_V (0 for r < 1e-6)."""
    r = torch.as_tensor(r, dtype=F64, device=alpha.device if torch.is_tensor(alpha) else None)
    safe = torch.where(r < 1e-6, torch.ones_like(r), r)
    if pol_form == 0:
        u6 = (safe / r_c) ** 6
        damp = 1.0 - torch.exp(-u6)
        v = -0.5 * alpha * damp * damp / safe ** 4
    else:
        v = -alpha / (2.0 * (safe * safe + r_c * r_c) ** 2)
    return torch.where(r < 1e-6, torch.zeros_like(v), v)


class _Energy:
    """Views, leaves and the small-stage graph of one energy."""

    def __init__(self, v, dr: float, device, orthogonalize: int, d_corr, spin, arrays=None):
        """v: an AdjView (or any object with its integer fields and E).  The
        inputs are the library's device buffers, or `arrays` (tensors in the
        same raw layouts: Rraw (n_window, Nt, Nt), Sraw, Graw (Nt, K) as
        leaves; VN, BN, BsN, CN, Bsw as matrices / raw windows)."""
        self.v = v
        self.dev = device
        N, ns, nw, Np, Nt, Nf, K, Npm = v.N, v.n_s, v.n_window, v.Np, v.Nt, v.Nf, v.Krows, v.Np_max
        self.E = v.E
        self.k = math.sqrt(2.0 * v.E)
        self.dr = dr
        if arrays is not None:
            self.Rraw = arrays["Rraw"].requires_grad_()
            self.Sraw = arrays["Sraw"].requires_grad_()
            self.Graw = arrays["Graw"].requires_grad_()
            self.VN = arrays["VN"].detach().clone().requires_grad_()
            self.BN, self.BsN, self.CN, self.Bsw = (arrays.get(x) for x in ("BN", "BsN", "CN", "Bsw"))
        else:
            # leaves: raw views of the window store and of G(N-1)^T (grads in the same layout)
            self.Rraw = _raw(v.Rwin, (nw, Nt, Nt), device).requires_grad_()
            self.Sraw = _raw(v.Swin, (nw, Np, Np), device).requires_grad_()
            self.Graw = _raw(v.G_last, (Nt, K), device).requires_grad_()
            VN = _raw(v.V_N, (Npm, Npm), device).T[:Np, :Np]
            self.VN = VN.detach().clone().requires_grad_()
            self.BN = _raw(v.B_N, (max(Nf, 1), Npm), device).T[:Np, :Nf] if Nf > 0 else None
            self.BsN = _raw(v.Bs_N, (max(Nf, 1), Npm), device).T[:Np, :Nf] if Nf > 0 else None
            self.CN = _raw(v.C_N, (Npm, K), device).T[:, :Np] if v.C_N else None
            self.Bsw = _raw(v.Bs_win, (nw, max(Nf, 1), Npm), device) if v.Bs_win else None
        self.orthogonalize = orthogonalize
        self.d_corr = torch.as_tensor(np.asarray(d_corr), dtype=F64, device=device)      # (6, n_occ)
        self.spin = torch.as_tensor(np.asarray(spin), dtype=F64, device=device)
        self.l_mu = np.array([int(math.isqrt(m)) for m in range(Np)])

    def _t(self, a):
        return torch.as_tensor(np.asarray(a, dtype=np.float64), dtype=F64, device=self.dev)

    def dipoles(self):
        """D of the six slots (6, Np) complex, from the views (with the graph)."""
        v = self.v
        N, ns, Np, Nt, Nf = v.N, v.n_s, v.Np, v.Nt, v.Nf
        h, dr, k, E = self.dr, self.dr, self.k, self.E
        h2_6, h2_12 = h * h / 6.0, h * h / 12.0
        Rw = lambda m: self.Rraw[m - ns].transpose(0, 1)
        Sw = lambda m: self.Sraw[m - ns].transpose(0, 1)
        # ---- K (KMatrixExtractor.cpp:75-198) at n_match = N - 1
        n_match = N - 1
        R = torch.linalg.inv(Rw(n_match))
        Rpp = R[:Np, :Np]
        if Nf > 0:
            Rpf, Rfp, Rff = R[:Np, Np:], R[Np:, :Np], R[Np:, Np:]
            coupled = not (float(torch.linalg.norm(Rpf.detach())) < 1e-14 and
                           float(torch.linalg.norm(Rfp.detach())) < 1e-14)
        else:
            coupled = False
        Ssch = Rpp - Rpf @ torch.linalg.inv(Rff) @ Rfp if coupled else Rpp
        Ssch = _sym(Ssch)
        l = self.l_mu
        lf = l.astype(np.float64)
        r_in, r_out = dr + n_match * h, dr + (n_match + 1) * h
        Jin = self._t([_rj(x, k * r_in) for x in l])
        Jout = self._t([_rj(x, k * r_out) for x in l])
        Yin = self._t([_ry(x, k * r_in) for x in l])
        Yout = self._t([_ry(x, k * r_out) for x in l])
        Win = self._t(1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_in * r_in)))
        Wout = self._t(1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_out * r_out)))
        A_mat = torch.diag(Wout * Jout) - Ssch * (Win * Jin)[None, :]
        B_mat = Ssch * (Win * Yin)[None, :] - torch.diag(Wout * Yout)
        K = _sym(torch.linalg.inv(B_mat) @ A_mat)
        self.K = K
        psi_N = torch.diag(Jout) + Yout[:, None] * K
        # ---- Z_N (BackPropagator.cpp:127-197) and the dipole contraction
        Zp = psi_N + (h2_6 * E) * psi_N - h2_6 * (self.VN @ psi_N)
        if N < v.n_tr and Nf > 0:
            fN = self.BN.T @ psi_N
            Zp = Zp - self.BsN @ fN
        Z = torch.cat([Zp, torch.zeros((Nt - Np, Np), dtype=F64, device=self.dev)], dim=0)
        Q = self.Graw.T @ Z
        if N < v.n_pts and self.CN is not None:
            Q = Q + self.CN @ psi_N
        # ---- the fit window, swept down from Z_N (BackPropagator.cpp:603-703)
        psi = {N: psi_N}
        for m in range(N - 1, ns - 1, -1):
            Z = Rw(m) @ Z
            if m < v.n_tr and Nf > 0:
                Bs = self.Bsw[m - ns].transpose(0, 1)[:Np, :Nf]
                psi[m] = Sw(m) @ (Z[:Np] - Bs @ Z[Np:])
            else:
                psi[m] = Sw(m) @ Z[:Np]
        # ---- fit (AsymptoticAmplitudes.cpp:64-359) over [n_s, ne_fit]
        ms = list(range(ns, v.ne_fit + 1))
        r = dr + np.array(ms, dtype=np.float64) * dr
        lmax = int(l.max()) if Np else 0
        jt = np.array([[_rj(L, k * x) for x in r] for L in range(lmax + 1)])
        yt = np.array([[_ry(L, k * x) for x in r] for L in range(lmax + 1)])
        c = np.zeros((lmax + 1, 4))
        closed = np.zeros(lmax + 1, dtype=bool)
        for L in range(lmax + 1):
            m00, m01, m11 = jt[L] @ jt[L], jt[L] @ yt[L], yt[L] @ yt[L]
            det = m00 * m11 - m01 * m01
            mx = max(abs(m00), abs(m01), abs(m11))
            if not (abs(det) > 1e-20 * mx * mx):
                closed[L] = True
            else:
                c[L] = [m11 / det, -m01 / det, -m01 / det, m00 / det]
        Pw = torch.stack([psi[m] for m in ms])                          # (nfit, Np, Np)
        YJ = torch.einsum("mi,imb->mb", self._t(jt[l]), Pw)
        YY = torch.einsum("mi,imb->mb", self._t(yt[l]), Pw)
        cm = self._t(c[l])
        A = cm[:, 0:1] * YJ + cm[:, 1:2] * YY
        B = cm[:, 2:3] * YJ + cm[:, 3:4] * YY
        cl = torch.as_tensor(closed[l], device=self.dev)[:, None]
        A = torch.where(cl, torch.eye(Np, dtype=F64, device=self.dev), A)
        B = torch.where(cl, torch.zeros_like(B), B)
        self.A, self.B = A, B
        # ---- dipoles (DipoleMatrixElement.cpp:920-947)
        M = torch.linalg.inv(A.to(torch.complex128) - 1j * B.to(torch.complex128)).conj().T
        Qc = Q.to(torch.complex128)
        Draw = (M @ Qc[:6].T).T                                          # (6, Np)
        if self.orthogonalize and Q.shape[0] > 6:
            o = (M @ Qc[6:].T).T                                         # (n_occ, Np)
            w = (self.spin[:, None] * self.d_corr.T).to(torch.complex128)    # (n_occ, 6)
            D = Draw - w.T @ o
        else:
            D = Draw
        return D


class ScanAdjoint:
    """Forward pass with checkpoints of a batch of energies (one l_cont),
    small stages in torch, and the library's reverse pass."""

    def __init__(self, solver: S.ScanSolver, energies, l_cont=None, segment: int = 256, opts=None):
        _bind()
        self.solver = solver
        E = np.ascontiguousarray(energies, dtype=np.float64).reshape(-1)
        self.energies = E
        nE = E.size
        lc = None
        if l_cont is not None:
            lc = np.ascontiguousarray(np.broadcast_to(np.asarray(l_cont, dtype=np.int32), (nE,)))
        self.opts = opts if opts is not None else S.default_opts(allow_closed_channels=1)
        arr, status, out = S.output_arrays(nE, solver.Np, solver.n_occ)
        self.h = C.c_void_p()
        code = lib().scatt_adjoint_forward(solver._ctx, C.byref(self.opts), nE, as_dptr(E),
                                           lc.ctypes.data_as(C.POINTER(C.c_int)) if lc is not None else None,
                                           int(segment), C.byref(out), C.byref(self.h))
        if code != 0:
            self.close()
            check(code)
        self.results = [S.result_of(arr, status, e, float(E[e]), int(lc[e]) if lc is not None else None, solver.Np)
                        for e in range(nE)]
        self.device = torch.device("cuda", solver.device)
        spin = np.full(solver.n_occ, 2.0)
        self.energy = []
        for i in range(nE):
            v = AdjView()
            check(lib().scatt_adjoint_view_of(self.h, i, C.byref(v)))
            self.energy.append(_Energy(v, solver.dr, self.device, self.opts.orthogonalize,
                                       self.results[i].d_corr, spin))
        self.Nr = self.energy[0].v.N + 1

    def dipoles(self):
        """[(6, Np) complex tensor] per energy, differentiable w.r.t. the views."""
        torch.cuda.synchronize(self.device)
        return [e.dipoles() for e in self.energy]

    def reverse(self, full: bool = False):
        """After backward() through the dipoles: the library's reverse pass.
        Returns (vtr (n_energy, Nr) numpy: tr dJ/dV(n) per energy, vfull:
        (Nr, Np_max, Np_max) tensor of dJ/dV(n) summed over the energies, or None)."""
        Npm = self.energy[0].v.Np_max
        vfull = torch.zeros((self.Nr, Npm, Npm), dtype=F64, device=self.device) if full else None
        vN = []
        for e in self.energy:
            v = e.v
            for leaf, ptr, shape in ((e.Rraw, v.RBwin, (v.n_window, v.Nt, v.Nt)),
                                     (e.Sraw, v.SBwin, (v.n_window, v.Np, v.Np)),
                                     (e.Graw, v.GB_last, (v.Nt, v.Krows))):
                dst = _raw(ptr, shape, self.device)
                if leaf.grad is None:
                    dst.zero_()
                else:
                    dst.copy_(leaf.grad)
            vN.append(e.VN.grad if e.VN.grad is not None else torch.zeros_like(e.VN))
        torch.cuda.synchronize(self.device)
        vtr = np.zeros((len(self.energy), self.Nr))
        check(lib().scatt_adjoint_reverse(self.h, as_dptr(vtr), C.c_void_p(vfull.data_ptr()) if full else None))
        N = self.Nr - 1
        for i, g in enumerate(vN):                 # V(N) enters only the outer boundary
            vtr[i, N] += float(torch.trace(g))
            if full:
                Np = g.shape[0]
                vfull[N].T[:Np, :Np] += g          # column-major per n, as the device writes
        return vtr, vfull

    def close(self):
        if getattr(self, "h", None):
            lib().scatt_adjoint_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _matrices(vfull):
    """dJ/dV(n) as matrices (the device stores them column-major per n)."""
    return vfull.transpose(1, 2)


class Dipoles(torch.autograd.Function):
    """D(alpha, r_c, dV) for a batch of energies of one l_cont, as a real
    (n_energy, 6, Np, 2) tensor (real, imaginary).

    alpha, r_c: 0-d float64 tensors (the V_pol parameters); dV: None or a
    symmetric (Nr, Np_max, Np_max) float64 CUDA tensor added to V(n); its
    gradient is the symmetrised dJ/dV(n)."""

    @staticmethod
    def forward(ctx, alpha, r_c, dV, solver, energies, pol_form=1, segment=256, opts=None):
        _bind()
        check(lib().scatt_set_polarization(solver._ctx, float(alpha), float(r_c), int(pol_form)))
        check(lib().scatt_set_potential_delta(solver._ctx, C.c_void_p(dV.data_ptr()) if dV is not None else None))
        try:
            adj = ScanAdjoint(solver, energies, segment=segment, opts=opts)
        finally:
            lib().scatt_set_potential_delta(solver._ctx, None)
        with torch.enable_grad():
            Ds = adj.dipoles()
            out = torch.stack([torch.view_as_real(D) for D in Ds])
        ctx.adj, ctx.out, ctx.pol_form = adj, out, int(pol_form)
        ctx.solver = solver
        # the reverse pass recomputes V(n) from the values of this forward
        # (V_pol parameters and dV are copied into the batch; dV's memory is
        # read again and must stay as it is until backward)
        ctx.dV = dV
        ctx.save_for_backward(alpha, r_c)
        ctx.has_dV = dV is not None
        return out.detach().clone()

    @staticmethod
    def backward(ctx, g):
        alpha, r_c = ctx.saved_tensors
        adj = ctx.adj
        with torch.enable_grad():
            torch.autograd.backward(ctx.out, g, retain_graph=True)
        need_full = ctx.needs_input_grad[2]
        vtr, vfull = adj.reverse(full=need_full)
        ga = gr = None
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            with torch.enable_grad():
                a = alpha.detach().clone().requires_grad_()
                rc = r_c.detach().clone().requires_grad_()
                n = torch.arange(adj.Nr, dtype=F64)
                vp = vpol(n * ctx.solver.dr, a, rc, ctx.pol_form)
                s = torch.sum(torch.as_tensor(vtr.sum(axis=0), dtype=F64) * vp)
                ga, gr = torch.autograd.grad(s, (a, rc), allow_unused=True)
        gdV = None
        if need_full:
            Vb = _matrices(vfull)
            gdV = 0.5 * (Vb + Vb.transpose(1, 2))
        return ga, gr, gdV, None, None, None, None, None


def observables(energies, D, e_homo: float, n_theta: int = 40, n_phi: int = 80):
    """The scan observables of scatt_b200.observables in torch, on D's device
    and inside the autograd graph, from D = Dipoles output (energies
    ascending): sigma_{length,velocity}_{x,y,z}, tau_* (two or more
    energies), q_{x,y,z}, dphi_rms_{x,y,z} and beta_{length,velocity}
    (postprocessing/cross_section_delay.py:195-430)."""
    Es = [float(x) for x in energies]
    k = torch.tensor([math.sqrt(2.0 * E) for E in Es], dtype=F64, device=D.device)
    om = torch.tensor([E - e_homo for E in Es], dtype=F64, device=D.device)
    Dc = torch.view_as_complex(D.contiguous())                           # (nE, 6, Np)
    out = {}
    for s in range(6):
        gauge = "length" if s < 3 else "velocity"
        pol = "xyz"[s % 3]
        Ds = Dc[:, s, :]
        s2 = torch.sum(torch.abs(Ds) ** 2, dim=1)
        if gauge == "length":
            out[f"sigma_{gauge}_{pol}"] = 8.0 * math.pi * om / (C_AU * k) * s2
        else:
            out[f"sigma_{gauge}_{pol}"] = 8.0 * math.pi / (C_AU * k * om) * s2
        if len(Es) > 1:
            out[f"tau_{gauge}_{pol}"] = torch.sum(torch.conj(Ds) * _d_dk(k, Ds) / k[:, None], dim=1).imag / s2
    for p, pol in enumerate("xyz"):
        DL, DV = Dc[:, p, :], Dc[:, 3 + p, :]
        sL, sV = torch.sum(torch.abs(DL) ** 2, dim=1), torch.sum(torch.abs(DV) ** 2, dim=1)
        out[f"q_{pol}"] = sV / (om ** 2 * sL)
        dphi = torch.angle(DV * torch.conj(DL))
        w = torch.abs(DL) * torch.abs(DV)
        out[f"dphi_rms_{pol}"] = torch.sqrt(torch.sum(w * dphi ** 2, dim=1) / torch.sum(w, dim=1))
    Y, weights, kx, ky, kz = _beta_grid(Dc.shape[2], n_theta, n_phi, D.device)
    for g, gauge in enumerate(("length", "velocity")):
        maps = [torch.tensordot(Dc[:, 3 * g + q, :], Y, dims=([1], [0])) for q in range(3)]
        sig = torch.sum((torch.abs(maps[0]) ** 2 + torch.abs(maps[1]) ** 2 + torch.abs(maps[2]) ** 2) * weights,
                        dim=(1, 2)) / 3.0
        n1 = torch.sum(torch.abs(maps[0] * kx + maps[1] * ky + maps[2] * kz) ** 2 * weights, dim=(1, 2))
        out[f"beta_{gauge}"] = n1 / sig - 1.0
    return out


def _beta_grid(n_ch: int, n_theta: int, n_phi: int, device):
    """Real Y_lm of channels 0 .. n_ch - 1 on the Gauss-Legendre (cos theta) x
    trapezoid (phi) grid of observables.beta, its weights and k-hat."""

    from .observables import real_ylm
    x, w = np.polynomial.legendre.leggauss(n_theta)
    theta = np.arccos(x)
    phi = np.arange(n_phi) * (2.0 * math.pi / n_phi)
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    Y = np.empty((n_ch, n_theta, n_phi))
    for mu in range(n_ch):
        l = math.isqrt(mu)
        Y[mu] = real_ylm(l, mu - l * l - l, TH, PH)
    t = lambda a: torch.tensor(a, dtype=F64, device=device)
    return (t(Y).to(torch.complex128), t(w[:, None] * (2.0 * math.pi / n_phi)),
            t(np.sin(TH) * np.cos(PH)), t(np.sin(TH) * np.sin(PH)), t(np.cos(TH)))


def _d_dk(k, f):
    """Second-order differences on an uneven grid along the first axis (numpy.gradient)."""
    n = k.shape[0]
    rows = [(f[1] - f[0]) / (k[1] - k[0])]
    for i in range(1, n - 1):
        hm, hp = k[i] - k[i - 1], k[i + 1] - k[i]
        rows.append((hm * hm * f[i + 1] - hp * hp * f[i - 1] + (hp * hp - hm * hm) * f[i]) / (hm * hp * (hm + hp)))
    rows.append((f[n - 1] - f[n - 2]) / (k[n - 1] - k[n - 2]))
    return torch.stack(rows)


__all__ = ["ScanAdjoint", "Dipoles", "observables", "vpol", "ScattError"]

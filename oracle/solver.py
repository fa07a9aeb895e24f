"""Per-energy scattering solve of the oracle (plain numpy / LAPACK).

Restates, stage by stage, the reference's run_one_energy (src/main.cpp:1081-1623):

  setup      WavefunctionSetup::prepare ......... WavefunctionSetup.cpp:219-376
  exchange   ExchangeCoupling ctor/compute_into . ExchangeCoupling.cpp:13-136
  Sinv       SchurInverter::build/compute_sinv_at SchurInverter.cpp:30-59, 247-415
  W^-1       WInverseOperator::apply/apply_U .... WInverseOperator.cpp:39-139
  FRP        ForwardRPropagator::run ............ ForwardRPropagator.cpp:49-134, 244-382
  KME        KMatrixExtractor::extract .......... KMatrixExtractor.cpp:75-224
  BP         BackPropagator::run ................ BackPropagator.cpp:127-197, 533-703
  AA         AsymptoticAmplitudes::extract ...... AsymptoticAmplitudes.cpp:64-359
  DME        DipoleMatrixElement::compute_six ... DipoleMatrixElement.cpp:49-282, 584-965

Dense inverses follow src/scatt/LapackInverse.hpp (MKL build):
inverse_general = dgetrf + dgetri (:53-92), inverse_symmetric_indefinite =
dsytrf + dsytri on the LOWER triangle, mirrored (:120-178).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
from scipy.linalg import lapack

from . import angular
from .bessel import riccati_j, riccati_y
from .potentials import VCube

W_MIN = 0.001          # SchurInverter.hpp:74
STAB_N_MAX = 60        # SchurInverter.hpp:75
SHIFT_MARGIN = 0.01    # SchurInverter.hpp:76
N_ASYM = 300           # main.cpp:1335
CHI_CUTOFF = 1e-15     # WavefunctionSetup.hpp:92


# ---------------------------------------------------------------- inverses
# The reference compiles src/scatt/LapackInverse.hpp two ways: with MKL
# (dgetrf/dgetri; dsytrf/dsytri on the LOWER triangle, mirrored) or without
# (Eigen partialPivLu().inverse(), plus 0.5 (M + M^T) for the "symmetric"
# variant, LapackInverse.hpp:88-91 and :166-176).  The oracle follows the
# Eigen build by default (BUILD = "eigen"); BUILD = "mkl" selects the MKL
# routines.  The two builds differ from each other by O(eps * cond) per step;
# on the synthetic H2- and H2O-like inputs that reaches ~2e-10 in K, which is
# the floor the GPU parity tolerances are set against.
BUILD = "eigen"


def inverse_general(A: np.ndarray) -> np.ndarray:
    """LapackInverse.hpp:53-92."""
    if BUILD == "mkl":
        lu, piv, info = lapack.dgetrf(A)
        if info != 0:
            raise np.linalg.LinAlgError(f"inverse_general: dgetrf failed (singular pivot), info = {info}")
        inv, info = lapack.dgetri(lu, piv)
        if info != 0:
            raise np.linalg.LinAlgError(f"inverse_general: dgetri failed, info = {info}")
        return inv
    # partial-pivot LU, then solve LU X = I (Eigen's partialPivLu().inverse())
    lu, piv, info = lapack.dgetrf(A)
    if info != 0:
        raise np.linalg.LinAlgError(f"inverse_general: singular pivot, info = {info}")
    inv, info = lapack.dgetrs(lu, piv, np.eye(A.shape[0]))
    return inv


def inverse_symmetric_indefinite(A: np.ndarray) -> np.ndarray:
    """LapackInverse.hpp:120-178."""
    if BUILD == "mkl":
        ldu, ipiv, info = lapack.dsytrf(A, lower=1)
        if info != 0:
            raise np.linalg.LinAlgError(f"inverse_symmetric_indefinite: dsytrf failed, info = {info}")
        inv, info = lapack.dsytri(ldu, ipiv, lower=1)
        if info != 0:
            raise np.linalg.LinAlgError(f"inverse_symmetric_indefinite: dsytri failed, info = {info}")
        return np.tril(inv) + np.tril(inv, -1).T
    inv = inverse_general(A)
    return 0.5 * (inv + inv.T)


def sym(M):
    return 0.5 * (M + M.T)


# ------------------------------------------------------- stability shift
def gershgorin_min(M):
    """SchurInverter.cpp:30-39."""
    off = np.sum(np.abs(M), axis=1) - np.abs(np.diag(M))
    return float(np.min(np.diag(M) - off))


def min_eig_fast(M, threshold):
    """SchurInverter.cpp:44-49 (eigen fallback reads the lower triangle)."""
    g = gershgorin_min(M)
    if g > threshold + 0.05:
        return g
    return float(sla.eigvalsh(M, lower=True)[0])


def shift_delta(M, W_min=W_MIN, margin=SHIFT_MARGIN) -> float:
    """SchurInverter.cpp:53-59: the diagonal shift for M, 0 when none."""
    me = min_eig_fast(M, W_min)
    return 0.0 if me >= W_min else W_min - me + margin


def stability_shift(M, W_min=W_MIN, margin=SHIFT_MARGIN, delta=None):
    """SchurInverter.cpp:53-59 -- returns (shifted M, shifted?).  delta:
    the shift decided elsewhere (on the whole matrix of a block solve)."""
    if delta is None:
        delta = shift_delta(M, W_min, margin)
    if delta == 0.0:
        return M, False
    M = M.copy()
    M[np.diag_indices_from(M)] += delta
    return M, True


# ------------------------------------------------------------ setup
@dataclass
class Setup:
    """Solver parameters and energy-independent tables (SolverParams + bundle)."""
    inp: object
    Nr: int
    dr: float
    l_cont: int
    l_x: int
    n_mu: int
    n_sigma: int
    n_lambda: int
    n_occ: int
    n_tr: int
    Nf: int
    Nt: int
    l_mu: np.ndarray
    m_mu: np.ndarray
    l_sigma_f: np.ndarray          # l of the sigma of each f channel (f = i*n_sigma + sigma)
    vcube: VCube
    Gc: sp.csr_matrix              # G_combined[(mu*n_sigma + sigma), lambda]
    n_lambda_max: int
    chi_r: np.ndarray              # (n_occ, n_lambda, n_tr): chi = r * F, r = ir*dr
    chi_init: np.ndarray           # (Nr, n_lambda) initial state (u-convention)
    phi: np.ndarray                # (n_occ, Nr, n_lambda) occupied orbitals
    spin: np.ndarray               # (n_occ,)
    mu_idx: np.ndarray | None = None   # continuum channels kept (full (l, m) indices), None: all
    whole: "Setup | None" = None       # block solves: the all-channel setup the shifts are decided on


def n_transition(inp, n_occ, n_lambda):
    """WavefunctionSetup.cpp:278-324 -- chi_cutoff scan + max(100, 5/dr) buffer."""
    F = inp.psi_lm[:n_occ, :min(n_lambda, inp.Nlm_store), :]
    mx = np.max(np.abs(F), axis=(0, 1))
    idx = np.nonzero(mx > CHI_CUTOFF)[0]
    last_ir = int(idx[-1]) if idx.size else 0
    buffer = max(100, int(5.0 / inp.dr))
    n_tr = min(inp.Nr, inp.Nr_store, last_ir + 1 + buffer)
    return max(1, n_tr)


def make_setup(inp, l_cont: int | None = None, vcube: VCube | None = None, channels=None,
               whole_matrix_shift: bool = True) -> Setup:
    """channels (optional): the continuum channels to keep, as full (l, m)
    indices l^2 + l + m <= (l_cont + 1)^2 - 1 -- a symmetry block.  The
    reference always keeps every channel; with a subset, V, the exchange
    rows and every per-channel table are those of the kept channels, the
    exchange channels all stay, and on a molecule whose potential and
    orbitals respect the symmetry the result is that block of the full
    solve.  The stability shifts (SchurInverter.cpp:53-59) are decided on
    the all-channel A and S, block-diagonal there, so on the lowest
    eigenvalue over every block, as a block-diagonal solve must to match the
    reference; whole_matrix_shift=False decides them on the block alone."""
    l_cont = inp.l_cont if l_cont is None else l_cont
    l_x = min(l_cont, 10)
    n_mu = (l_cont + 1) ** 2
    n_sigma = (l_x + 1) ** 2
    n_lambda = (l_cont + l_x + 1) ** 2
    n_occ = inp.n_occ
    Nr, dr = inp.Nr, inp.dr
    n_tr = n_transition(inp, n_occ, n_lambda)
    lm = [angular.idx_to_lm(i) for i in range(n_mu)]
    ls = np.array([angular.idx_to_lm(s)[0] for s in range(n_sigma)])
    Nf = n_occ * n_sigma
    G = angular.build_G_vector(n_mu, n_lambda, n_sigma)
    # ExchangeCoupling.cpp:28-53
    nlm = 0
    for a, b, c, v in G:
        if a < n_mu and c < n_sigma and b + 1 > nlm:
            nlm = b + 1
    rows = [a * n_sigma + c for a, b, c, v in G if b < nlm]
    cols = [b for a, b, c, v in G if b < nlm]
    vals = [v for a, b, c, v in G if b < nlm]
    Gc = sp.csr_matrix((vals, (rows, cols)), shape=(n_mu * n_sigma, max(nlm, 1)))
    Gc.sum_duplicates()
    Gc.sort_indices()
    mu_idx = None
    if channels is not None:
        mu_idx = np.array(sorted(set(int(c) for c in channels)), dtype=np.int64)
        if mu_idx.size == 0 or mu_idx[0] < 0 or mu_idx[-1] >= n_mu:
            raise ValueError("channels must be non-empty full (l, m) indices below (l_cont + 1)^2")
        Gc = Gc[(mu_idx[:, None] * n_sigma + np.arange(n_sigma)[None, :]).ravel()]
        lm = [lm[i] for i in mu_idx]
        n_mu = int(mu_idx.size)
    # chi[ir](i, lambda) = r * psi_lm, r = rmin + ir*dr, rmin = 0 (WavefunctionSetup.cpp:196-204)
    nl = min(n_lambda, inp.Nlm_store)
    chi_r = np.zeros((n_occ, n_lambda, n_tr))
    r = np.arange(n_tr) * dr
    chi_r[:, :nl, :] = inp.psi_lm[:n_occ, :nl, :n_tr] * r[None, None, :]
    # main.cpp:767-822: occupied orbitals (target) and the initial state
    phi = np.zeros((n_occ, Nr, n_lambda))
    phi[:, :n_tr, :] = np.transpose(chi_r, (0, 2, 1))
    init = inp.init_state if inp.init_state >= 0 else n_occ - 1
    chi_init = np.zeros((Nr, n_lambda))
    if init < n_occ:
        chi_init[:, :] = phi[init]
    else:
        ntake = min(n_tr, inp.Nr_store)
        chi_init[:ntake, :nl] = (inp.psi_lm[init, :nl, :ntake] * (np.arange(ntake) * dr)[None, :]).T
    spin = np.full(n_occ, 2.0)
    if vcube is None:
        vcube = VCube(inp)
    whole = make_setup(inp, l_cont, vcube) if (mu_idx is not None and whole_matrix_shift) else None
    return Setup(inp, Nr, dr, l_cont, l_x, n_mu, n_sigma, n_lambda, n_occ, n_tr, Nf, n_mu + Nf,
                 np.array([a for a, b in lm]), np.array([b for a, b in lm]),
                 np.tile(ls, n_occ), vcube, Gc, nlm, chi_r, chi_init, phi, spin, mu_idx, whole)


def V_at(st: Setup, n: int) -> np.ndarray:
    if st.mu_idx is not None:
        return st.vcube.get(n)[np.ix_(st.mu_idx, st.mu_idx)]
    return st.vcube.get(n)[: st.n_mu, : st.n_mu]


# ----------------------------------------------------- exchange coupling
def exchange_Q(st: Setup, ir: int) -> np.ndarray:
    """ExchangeCoupling.cpp:65-136 -- Q_psi_f(r_ir), r = ir*dr (rmin = 0)."""
    Q = np.zeros((st.n_mu, st.Nf))
    r = ir * st.dr
    if r < 1e-10 or ir >= st.n_tr or st.n_lambda_max == 0:
        return Q
    factor = 2.0 * math.sqrt(2.0 * math.pi) / r
    chiT = st.chi_r[:, : st.n_lambda_max, ir].T          # (n_lambda_max, n_occ)
    Qf = st.Gc @ chiT                                      # (n_mu*n_sigma, n_occ)
    Qf = Qf.reshape(st.n_mu, st.n_sigma, st.n_occ)
    for i in range(st.n_occ):
        Q[:, i * st.n_sigma:(i + 1) * st.n_sigma] = factor * Qf[:, :, i]
    return Q


def dinv_at(st: Setup, n: int, W_min=W_MIN) -> np.ndarray:
    """SchurInverter.cpp:332-339 / WInverseOperator.cpp:45-52, r = (n+1)*dr."""
    r = st.dr + n * st.dr
    r2 = r * r
    h2_12 = st.dr * st.dr / 12.0
    l = st.l_sigma_f.astype(np.float64)
    cent = np.where(r2 > 1e-30, (l * (l + 1.0)) / r2, 0.0)
    Df = 1.0 - h2_12 * cent
    Df = np.where(Df < W_min, W_min, Df)
    return 1.0 / Df


def B_at(st: Setup, n: int) -> np.ndarray:
    """WInverseOperator.cpp:54-61 -- B = h^2/12 Q (zero past n_transition)."""
    if n >= st.n_tr:
        return np.zeros((st.n_mu, st.Nf))
    return (st.dr * st.dr / 12.0) * exchange_Q(st, n)


# ------------------------------------------------------------ Sinv
def sinv_at(st: Setup, E: float, n: int, counts=None) -> np.ndarray:
    """SchurInverter.cpp:247-415 (CPU path, use_symmetric_inverse = true)."""
    h2_6 = st.dr * st.dr / 6.0
    A = np.eye(st.n_mu)
    A[np.diag_indices(st.n_mu)] += h2_6 * E
    if n < st.Nr:
        A = A - h2_6 * V_at(st, n)
    d_A = d_S = None
    if st.whole is not None and n < STAB_N_MAX:
        d_A, d_S = whole_shifts(st.whole, E, n)
    if n < STAB_N_MAX:
        A = sym(A)
        A, sh = stability_shift(A, delta=d_A)
        if counts is not None and sh:
            counts["A"] += 1
    if n < st.n_tr:
        Dinv = dinv_at(st, n)
        B = B_at(st, n)
        Bs = B * Dinv[None, :]
        S = A - Bs @ B.T
        if n < STAB_N_MAX:
            S, sh = stability_shift(S, delta=d_S)
            if counts is not None and sh:
                counts["S"] += 1
    else:
        S = A
    return inverse_symmetric_indefinite(S)


def whole_shifts(st: Setup, E: float, n: int):
    """The shifts of A and S that sinv_at applies at n on the all-channel
    setup st: (delta_A, delta_S), 0 where none."""
    h2_6 = st.dr * st.dr / 6.0
    A = np.eye(st.n_mu)
    A[np.diag_indices(st.n_mu)] += h2_6 * E
    if n < st.Nr:
        A = A - h2_6 * V_at(st, n)
    d_A = shift_delta(sym(A))
    d_S = 0.0
    if n < st.n_tr:
        A, _ = stability_shift(sym(A), delta=d_A)
        B = B_at(st, n)
        d_S = shift_delta(A - (B * dinv_at(st, n)[None, :]) @ B.T)
    return d_A, d_S


# ------------------------------------------------------------ W^-1
def winv_apply(st: Setup, n: int, Sinv: np.ndarray, Z: np.ndarray) -> np.ndarray:
    """WInverseOperator.cpp:75-128."""
    Dinv = dinv_at(st, n)
    Zp, Zf = Z[: st.n_mu], Z[st.n_mu:]
    tmp_f = Dinv[:, None] * Zf
    exch = n < st.n_tr
    if exch:
        B = B_at(st, n)
        rhs = Zp - B @ tmp_f
    else:
        rhs = Zp
    Y = np.empty_like(Z)
    Y[: st.n_mu] = Sinv @ rhs
    if exch:
        Y[st.n_mu:] = tmp_f - Dinv[:, None] * (B.T @ Y[: st.n_mu])
    else:
        Y[st.n_mu:] = tmp_f
    return Y


# ------------------------------------------------------------ FRP
def n_start(st: Setup) -> int:
    """ForwardRPropagator.cpp:49-62."""
    lmf = st.l_x
    r_crit = st.dr * math.sqrt(float(lmf * (lmf + 1)) / 12.0)
    ns = max(1, int(math.ceil(2.0 * r_crit / st.dr)))
    return min(ns, st.Nr - 1)


def analytic_init(st: Setup, E: float, n: int, W_min=W_MIN) -> np.ndarray:
    """ForwardRPropagator.cpp:78-134 -- diagonal Rinv for 1 <= n < n_start."""
    R = np.zeros((st.Nt, st.Nt))
    if n <= 0:
        return R
    h = st.dr
    h2_12, h2_6 = h * h / 12.0, h * h / 6.0
    k = math.sqrt(2.0 * E)
    rn, rn1 = st.dr + n * h, st.dr + (n + 1) * h
    Vn, Vn1 = V_at(st, n), V_at(st, n + 1)
    for mu in range(st.n_mu):
        Mn = 1.0 + h2_6 * (E - Vn[mu, mu])
        Mn1 = 1.0 + h2_6 * (E - Vn1[mu, mu])
        yn = riccati_j(int(st.l_mu[mu]), k * rn)
        yn1 = riccati_j(int(st.l_mu[mu]), k * rn1)
        den = Mn1 * yn1
        if abs(den) > 1e-300:
            R[mu, mu] = (Mn * yn) / den
    rn2, rn12 = rn * rn, rn1 * rn1
    for f in range(st.Nf):
        l = int(st.l_sigma_f[f])
        cn = (l * (l + 1)) / rn2 if rn2 > 1e-30 else 0.0
        cn1 = (l * (l + 1)) / rn12 if rn12 > 1e-30 else 0.0
        Mn = 1.0 - h2_12 * cn
        Mn1 = 1.0 - h2_12 * cn1
        Mn = W_min if Mn < W_min else Mn
        Mn1 = W_min if Mn1 < W_min else Mn1
        yn = rn ** float(l + 1)
        yn1 = rn1 ** float(l + 1)
        den = Mn1 * yn1
        if abs(den) > 1e-300:
            R[st.n_mu + f, st.n_mu + f] = (Mn * yn) / den
    return R


def frp_step(st: Setup, n: int, Sinv: np.ndarray, Rinv_prev: np.ndarray) -> np.ndarray:
    """ForwardRPropagator.cpp:332-358 (CPU path)."""
    I = np.eye(st.Nt)
    U = 12.0 * winv_apply(st, n, Sinv, I) - 10.0 * I
    R = U - Rinv_prev
    return sym(inverse_general(R))


# ------------------------------------------------------------ KME
def kme_extract(st: Setup, E: float, Rinv_nM: np.ndarray, n_match: int):
    """KMatrixExtractor.cpp:75-198."""
    Np, Nf = st.n_mu, st.Nf
    h = st.dr
    h2_12 = h * h / 12.0
    k = math.sqrt(2.0 * E)
    r_in = st.dr + n_match * h
    r_out = st.dr + (n_match + 1) * h
    R = inverse_general(Rinv_nM)
    Rpp, Rpf, Rfp, Rff = R[:Np, :Np], R[:Np, Np:], R[Np:, :Np], R[Np:, Np:]
    coupling_zero = False
    if Nf == 0:
        S = R
        coupling_zero = True
    elif np.linalg.norm(Rpf) < 1e-14 and np.linalg.norm(Rfp) < 1e-14:
        S = Rpp
        coupling_zero = True
    else:
        S = Rpp - Rpf @ inverse_general(Rff) @ Rfp
    S = sym(S)
    l = st.l_mu
    Jin, Jout = riccati_j(l, k * r_in), riccati_j(l, k * r_out)
    Yin, Yout = riccati_y(l, k * r_in), riccati_y(l, k * r_out)
    lf = l.astype(np.float64)
    Win = 1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_in * r_in))
    Wout = 1.0 + h2_12 * (k * k - lf * (lf + 1.0) / (r_out * r_out))
    A_mat = np.diag(Wout * Jout) - S @ np.diag(Win * Jin)
    B_mat = S @ np.diag(Win * Yin) - np.diag(Wout * Yout)
    lu = sla.lu_factor(B_mat)
    K = sym(sla.lu_solve(lu, A_mat))
    I = np.eye(Np)
    Smat = (I + 1j * K) @ np.linalg.inv(I - 1j * K)
    out = dict(K=K, S=Smat, K_symmetry_err=float(np.max(np.abs(K - K.T))),
               unitarity_err=float(np.max(np.abs(Smat.conj().T @ Smat - I))),
               eigenphases=np.arctan(sla.eigvalsh(K, lower=True)),
               schur_coupling_zero=coupling_zero, n_match=n_match)
    return out


def psi_boundary(st: Setup, E: float, K: np.ndarray) -> np.ndarray:
    """KMatrixExtractor.cpp:201-224 -- J_N + N_N K at r_N = r_min + (Nr-1) dr."""
    k = math.sqrt(2.0 * E)
    rN = st.dr + (st.Nr - 1) * st.dr
    J = riccati_j(st.l_mu, k * rN)
    Y = riccati_y(st.l_mu, k * rN)
    return np.diag(J) + Y[:, None] * K


# ------------------------------------------------------------ AA
def aa_window(st: Setup):
    """AsymptoticAmplitudes.cpp:70-91 with the BP asym buffer [N-299, N]."""
    Nr = st.Nr
    N = Nr - 1
    ns = max(Nr - 200, int(0.9 * Nr))
    ne = Nr - 1 - 3
    lo = N - N_ASYM + 1
    ns, ne = max(ns, lo), min(ne, N)
    if ne - ns + 1 < 10:
        raise RuntimeError("AsymptoticAmplitudes: fit window is too small")
    return ns, ne


def aa_extract(st: Setup, E: float, psi_tail: dict, allow_closed=True):
    """AsymptoticAmplitudes.cpp:64-359."""
    Np = st.n_mu
    k = math.sqrt(2.0 * E)
    ns, ne = aa_window(st)
    nfit = ne - ns + 1
    r = st.dr + np.arange(ns, ne + 1) * st.dr
    uls = sorted(set(int(x) for x in st.l_mu))
    jh = {l: riccati_j(l, k * r) for l in uls}
    yh = {l: riccati_y(l, k * r) for l in uls}
    closed, Minv = {}, {}
    for l in uls:
        M = np.array([[jh[l] @ jh[l], jh[l] @ yh[l]], [jh[l] @ yh[l], yh[l] @ yh[l]]])
        det = M[0, 0] * M[1, 1] - M[0, 1] * M[1, 0]
        mx = np.max(np.abs(M))
        singular = not (abs(det) > 1e-20 * mx * mx)
        if singular:
            if not allow_closed:
                raise RuntimeError(f"AsymptoticAmplitudes: singular normal matrix for l={l}")
            closed[l] = True
        else:
            closed[l] = False
            Minv[l] = np.linalg.inv(M)
    Jc = np.array([jh[int(l)] for l in st.l_mu])
    Yc = np.array([yh[int(l)] for l in st.l_mu])
    YJ = np.zeros((Np, Np))
    YY = np.zeros((Np, Np))
    max_psi = 0.0
    for i in range(nfit):
        p = psi_tail[ns + i]
        max_psi = max(max_psi, float(np.max(np.abs(p))))
        YJ += Jc[:, i:i + 1] * p
        YY += Yc[:, i:i + 1] * p
    A = np.zeros((Np, Np))
    B = np.zeros((Np, Np))
    mu_closed = np.array([closed[int(l)] for l in st.l_mu])
    for mu in range(Np):
        l = int(st.l_mu[mu])
        if closed[l]:
            A[mu, mu] = 1.0
            continue
        Mi = Minv[l]
        A[mu] = Mi[0, 0] * YJ[mu] + Mi[0, 1] * YY[mu]
        B[mu] = Mi[1, 0] * YJ[mu] + Mi[1, 1] * YY[mu]
    max_res = 0.0
    for i in range(nfit):
        fit = Jc[:, i:i + 1] * A + Yc[:, i:i + 1] * B
        d = np.abs(fit - psi_tail[ns + i])
        d[mu_closed] = 0.0
        max_res = max(max_res, float(np.max(d)))
    K = B @ np.linalg.inv(A)
    Smat = (A + 1j * B) @ np.linalg.inv(A - 1j * B)
    I = np.eye(Np)
    return dict(A=A, B=B, K=K, S=Smat,
                fit_residual_max=max_res, fit_residual_rel=max_res / max(max_psi, 1e-30),
                A_minus_I_max=float(np.max(np.abs(A - I))),
                K_symmetry_err=float(np.max(np.abs(K - K.T))),
                S_unitarity_err=float(np.max(np.abs(Smat.conj().T @ Smat - I))),
                eigenphases=np.arctan(sla.eigvalsh(K, lower=True)),
                n_fit_start=ns, n_fit_end=ne, closed_l=[l for l in uls if closed[l]])


# ------------------------------------------------------------ DME
def five_point_derivative(f: np.ndarray, dr: float) -> np.ndarray:
    """DipoleMatrixElement.cpp:49-74."""
    n = f.shape[0]
    df = np.zeros_like(f)
    if n < 5:
        if n >= 2:
            df[0] = (f[1] - f[0]) / dr
            df[1:n - 1] = (f[2:] - f[:-2]) / (2.0 * dr)
            df[n - 1] = (f[n - 1] - f[n - 2]) / dr
        return df
    c = 1.0 / (12.0 * dr)
    df[2:n - 2] = (-f[4:] + 8.0 * f[3:n - 1] - 8.0 * f[1:n - 3] + f[:n - 4]) * c
    df[0] = (-25.0 * f[0] + 48.0 * f[1] - 36.0 * f[2] + 16.0 * f[3] - 3.0 * f[4]) * c
    df[1] = (-3.0 * f[0] - 10.0 * f[1] + 18.0 * f[2] - 6.0 * f[3] + 1.0 * f[4]) * c
    df[n - 2] = (-1.0 * f[n - 5] + 6.0 * f[n - 4] - 18.0 * f[n - 3] + 10.0 * f[n - 2] + 3.0 * f[n - 1]) * c
    df[n - 1] = (3.0 * f[n - 5] - 16.0 * f[n - 4] + 36.0 * f[n - 3] - 48.0 * f[n - 2] + 25.0 * f[n - 1]) * c
    return df


def simpson(f: np.ndarray, h: float) -> np.ndarray:
    """DipoleMatrixElement.cpp:142-192 along the last axis (1/3 rule; 3/8 on the last 4 points)."""
    n = f.shape[-1]
    if n < 2:
        return np.zeros(f.shape[:-1])

    def one_third(m):
        s = f[..., 0] + f[..., m - 1]
        s = s + 4.0 * np.sum(f[..., 1:max(m - 1, 0):2], axis=-1)
        s = s + 2.0 * np.sum(f[..., 2:max(m - 2, 0):2], axis=-1)
        return s * h / 3.0

    if n == 2:
        return 0.5 * h * (f[..., 0] + f[..., 1])
    if n % 2 == 1:
        return one_third(n)
    if n < 4:
        s = 0.5 * (f[..., 0] + f[..., n - 1]) + np.sum(f[..., 1:n - 1], axis=-1)
        return s * h
    return one_third(n - 3) + (3.0 * h / 8.0) * (f[..., n - 4] + 3.0 * f[..., n - 3]
                                                 + 3.0 * f[..., n - 2] + f[..., n - 1])


SLOTS = [("L", 1), ("L", -1), ("L", 0), ("V", 1), ("V", -1), ("V", 0)]   # DipoleMatrixElement.cpp:603-610


def angular_table(st: Setup, q: int) -> np.ndarray:
    """DipoleMatrixElement.cpp:628-640."""
    Nl = st.n_lambda
    Ang = np.zeros((st.n_mu, Nl))
    lnu = [angular.idx_to_lm(nu) for nu in range(Nl)]
    for mu in range(st.n_mu):
        lmu, mmu = int(st.l_mu[mu]), int(st.m_mu[mu])
        for nu, (ln, mn) in enumerate(lnu):
            if abs(lmu - ln) != 1:
                continue
            a = angular.angular_dipole(lmu, mmu, q, ln, mn)
            if a != 0.0:
                Ang[mu, nu] = a
    return Ang


def xi_tables(st: Setup, n_lo: int, n_hi: int):
    """DipoleMatrixElement.cpp:204-233 -- Xi_slot(row, mu) for the 6 slots."""
    dchi = np.stack([five_point_derivative(st.chi_init[:, nu], st.dr)
                     for nu in range(st.n_lambda)], axis=1)
    rows = np.arange(n_lo, n_hi)
    r = st.dr + rows * st.dr
    inv_r = np.where(r > 1e-30, 1.0 / r, 0.0)
    lnu = np.array([angular.idx_to_lm(nu)[0] for nu in range(st.n_lambda)])
    out = []
    angs = {q: angular_table(st, q) for q in (1, -1, 0)}
    for g, q in SLOTS:
        Ang = angs[q]
        if g == "L":
            Xi = st.chi_init[rows] @ Ang.T
        else:
            Xi = np.zeros((rows.size, st.n_mu))
            for mu in range(st.n_mu):
                c = np.array([angular.velocity_coef(int(st.l_mu[mu]), int(ln)) for ln in lnu])
                Xi[:, mu] = (dchi[rows] + (c[None, :] * inv_r[:, None]) * st.chi_init[rows]) @ Ang[mu]
        out.append(Xi)
    return out


def dme_compute_six(st: Setup, A, B, psi_of, n_lo: int, n_hi: int, orthogonalize=True):
    """DipoleMatrixElement.cpp:584-965 -- 6 slices (L/V x x/y/z) plus b_overlap."""
    n_pts = n_hi - n_lo
    if n_pts < 5:
        raise RuntimeError("DipoleMatrixElement: too few radial points for integration")
    Np = st.n_mu
    Xi = xi_tables(st, n_lo, n_hi)
    M = np.linalg.inv(A.astype(complex) - 1j * B.astype(complex)).conj().T
    rows = np.arange(n_lo, n_hi)
    r = st.dr + rows * st.dr
    integ = np.zeros((6, Np, n_pts))
    bint = np.zeros((st.n_occ, Np, n_pts))
    mu_hi = min(Np, st.n_lambda)
    for row, ir in enumerate(rows):
        p = psi_of(ir)
        for s, (g, q) in enumerate(SLOTS):
            rfac = r[row] if g == "L" else 1.0
            integ[s, :, row] = rfac * (Xi[s][row] @ p)
        if orthogonalize:
            for a in range(st.n_occ):
                bint[a, :, row] = st.phi[a, ir, :mu_hi] @ p[:mu_hi]
    b_overlap = simpson(bint, st.dr).T if orthogonalize else None      # (Np, n_occ)
    res = []
    for s, (g, q) in enumerate(SLOTS):
        d_raw = simpson(integ[s], st.dr)
        D_raw = M @ d_raw.astype(complex)
        if not orthogonalize:
            res.append(dict(d_raw=d_raw, D_raw=D_raw, D=D_raw, d_corr=np.zeros(0),
                            partial_sigma=float(np.sum(np.abs(D_raw) ** 2))))
            continue
        rfac = r if g == "L" else np.ones_like(r)
        dcorr = np.array([simpson(rfac * np.sum(st.phi[a, rows, :mu_hi] * Xi[s][:, :mu_hi], axis=1), st.dr)
                          for a in range(st.n_occ)])
        o = M @ b_overlap.astype(complex)
        D = D_raw - o @ (st.spin * dcorr)
        res.append(dict(d_raw=d_raw, D_raw=D_raw, D=D, d_corr=dcorr,
                        partial_sigma=float(np.sum(np.abs(D) ** 2))))
    return res, b_overlap


# ------------------------------------------------------------ driver
@dataclass
class EnergyResult:
    E: float
    K_kme: np.ndarray
    kme: dict
    aa: dict
    slices: list
    b_overlap: np.ndarray
    psi_keep: dict = field(default_factory=dict)
    rinv: list | None = None
    shifts: dict = field(default_factory=dict)


def solve_energy(st: Setup, E: float, keep_rinv=False, keep_psi=False) -> EnergyResult:
    """run_one_energy (main.cpp:1124-1611) for one energy, all stages on the CPU."""
    Nr, Nt, Np = st.Nr, st.Nt, st.n_mu
    counts = {"A": 0, "S": 0}
    ns = n_start(st)
    # SchurInverter::build -- Sinv for all n (stored)
    Sinv = [sinv_at(st, E, n, counts) for n in range(Nr)]
    # ForwardRPropagator::run
    Rinv = [None] * Nr
    for n in range(ns):
        Rinv[n] = analytic_init(st, E, n)
    prev = Rinv[ns - 1]
    for n in range(ns, Nr):
        prev = frp_step(st, n, Sinv[n], prev)
        Rinv[n] = prev
    # KMatrixExtractor
    n_match = Nr - 2
    kme = kme_extract(st, E, Rinv[n_match], n_match)
    bc = psi_boundary(st, E, kme["K"])
    # BackPropagator::run (BackPropagator.cpp:533-703)
    N = Nr - 1
    n_keep_hi = min(Nr - 1, max(1, st.n_tr - 1))
    asym_lo = N - N_ASYM + 1
    Dinv_N = dinv_at(st, N)
    B_N = B_at(st, N)
    f_N = -(Dinv_N[:, None] * (B_N.T @ bc))
    h2_6 = st.dr * st.dr / 6.0
    Z = np.zeros((Nt, Np))
    Z[:Np] = bc + h2_6 * E * bc - h2_6 * V_at(st, N) @ bc + B_N @ f_N
    psi = {}
    if N <= n_keep_hi or N >= asym_lo:
        psi[N] = bc
    for n in range(N - 1, -1, -1):
        Z = Rinv[n] @ Z
        Y = winv_apply(st, n, Sinv[n], Z)
        if n <= n_keep_hi or n >= asym_lo:
            psi[n] = Y[:Np].copy()
    # AsymptoticAmplitudes
    aa = aa_extract(st, E, psi)
    # DipoleMatrixElement::compute_six over [0, n_keep_hi]
    n_hi = min(Nr, n_keep_hi + 1)
    slices, b_overlap = dme_compute_six(st, aa["A"], aa["B"], lambda ir: psi[ir], 0, n_hi)
    return EnergyResult(E, kme["K"], kme, aa, slices, b_overlap,
                        psi_keep=psi if keep_psi else {}, rinv=Rinv if keep_rinv else None,
                        shifts=counts)


def solve_energy_lean(st: Setup, E: float, seg: int = 256, psi_dir: str | None = None) -> EnergyResult:
    """solve_energy with bounded memory, for the full-size grids.

    The same stage functions in the same order as solve_energy, so the same
    arithmetic: the forward recurrence keeps Rinv only at segment ends (every
    `seg` steps) and the backward sweep recomputes each segment's Sinv and
    Rinv from its checkpoint before walking it downward, as the reference's
    checkpointed stages do when R^-1 does not fit in memory
    (ForwardRPropagator.cpp:244-382, BackPropagator.cpp:533-703).  psi over
    [0, n_transition) -- 1.56 MB a point at l_cont = 20 -- goes to a
    disk-backed array under psi_dir (a temporary directory by default).
    """
    import os
    import tempfile
    Nr, Nt, Np = st.Nr, st.Nt, st.n_mu
    counts = {"A": 0, "S": 0}
    ns = n_start(st)

    def rinv_range(a, b, prev, cnt=None):
        """Sinv(n), Rinv(n) for n in [a, b), from Rinv(a-1) = prev."""
        S, R = {}, {}
        for n in range(a, b):
            S[n] = sinv_at(st, E, n, cnt)
            if n < ns:
                R[n] = analytic_init(st, E, n)
            else:
                R[n] = frp_step(st, n, S[n], prev)
            prev = R[n]
        return S, R

    ck = {}                      # ck[a] = Rinv(a - 1), the state entering segment [a, a + seg)
    prev = None
    keep_match = None
    n_match = Nr - 2
    for a in range(0, Nr, seg):
        b = min(Nr, a + seg)
        ck[a] = prev
        _, R = rinv_range(a, b, prev, counts)
        prev = R[b - 1]
        if a <= n_match < b:
            keep_match = R[n_match]
    kme = kme_extract(st, E, keep_match, n_match)
    bc = psi_boundary(st, E, kme["K"])
    N = Nr - 1
    n_keep_hi = min(Nr - 1, max(1, st.n_tr - 1))
    asym_lo = N - N_ASYM + 1
    Dinv_N = dinv_at(st, N)
    B_N = B_at(st, N)
    f_N = -(Dinv_N[:, None] * (B_N.T @ bc))
    h2_6 = st.dr * st.dr / 6.0
    Z = np.zeros((Nt, Np))
    Z[:Np] = bc + h2_6 * E * bc - h2_6 * V_at(st, N) @ bc + B_N @ f_N
    tmp = tempfile.mkdtemp(dir=psi_dir)
    store = np.lib.format.open_memmap(os.path.join(tmp, "psi.npy"), mode="w+",
                                      dtype=np.float64, shape=(n_keep_hi + 1, Np, Np))
    psi = {}

    def keep(n, p):
        if n <= n_keep_hi:
            store[n] = p
        if n >= asym_lo:
            psi[n] = p.copy()

    keep(N, bc)
    starts = sorted(ck)
    for a in reversed(starts):
        b = min(Nr, a + seg)
        lo_n, hi_n = a, min(b, N)           # the sweep visits n = N-1 .. 0
        if lo_n >= hi_n:
            continue
        S, R = rinv_range(a, b, ck[a])
        for n in range(hi_n - 1, lo_n - 1, -1):
            Z = R[n] @ Z
            Y = winv_apply(st, n, S[n], Z)
            keep(n, Y[:Np])
        del S, R
    aa = aa_extract(st, E, psi)
    n_hi = min(Nr, n_keep_hi + 1)
    slices, b_overlap = dme_compute_six(st, aa["A"], aa["B"], lambda ir: store[ir], 0, n_hi)
    del store
    try:
        os.remove(os.path.join(tmp, "psi.npy"))
        os.rmdir(tmp)
    except OSError:
        pass
    return EnergyResult(E, kme["K"], kme, aa, slices, b_overlap, shifts=counts)

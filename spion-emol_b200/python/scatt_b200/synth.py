"""Seeded synthetic molecular inputs with the shapes of the benchmark systems.

The reference reads its inputs from a preprocessing HDF5 file (orbital
single-centre expansions psi_lm, the Hartree multipoles V_H, the atoms;
src/io/HDF5Reader.hpp:42-86).  No such file exists here, so these
generators build inputs of the same shapes, sizes and value distributions:

* ``h2_like``      two Z=1 centres at z = +-0.7 bohr, one doubly occupied
                   sigma_g orbital chi_l(r) = c_l r^(l+1) exp(-1.2 r),
                   even l <= 8, m = 0, seeded Gaussian c_l, unit norm.
* ``h2o_like``     O (Z=8) at the origin and two H at 1.81 bohr / 104.5 deg,
                   five doubly occupied orbitals with seeded
                   r^(l+1) exp(-zeta_l r) envelopes up to lmax, Gram-Schmidt
                   orthonormalised on the grid.
* ``c8f8_like``    eight C and eight F on a jittered cubane-like frame.

Radial functions are stored the way the HDF5 stores them: psi_lm = F(r)
(so chi = r * F), sampled at r = ir * dr (the preprocessing grid starts at
r = 0).  V_H is the radial-Poisson potential of the spherically averaged
electron density (the L = 0 Hartree multipole); higher Hartree multipoles
are left out of the synthetic input.  The nuclear multipoles V_en are not
part of the input: the solver builds them from the atoms, as the reference
does (src/scatt/Potentials.cpp:40-88).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SEED_BASE = 20261203
BOHR_PER_ANGSTROM = 1.0 / 0.529177210903


def lm_to_idx(l: int, m: int) -> int:
    return l * l + l + m


@dataclass
class ScanInputs:
    """Energy-independent inputs of one scan (what the preprocessing file holds)."""
    name: str
    dr: float
    Nr: int
    l_cont: int
    atoms: np.ndarray            # (n_atoms, 4): Z, x, y, z  [bohr]
    psi_lm: np.ndarray           # (n_orb, Nlm_store, Nr_store): F_{i,lambda}(r_ir)
    orb_energies: np.ndarray     # (n_orb,)
    n_occ: int                   # occupied orbitals in the exchange sum
    V_H: np.ndarray              # (n_H, Nr): Hartree multipoles V_H,sigma(r_ir)
    alpha_pol: float = 0.0       # polarisability (0 -> no V_pol)
    pol_form: int = 0            # 0: reference damped form, 1: -a/(2(r^2+rc^2)^2)
    r_c: float = 1.5
    init_state: int = -1         # orbital used as the dipole initial state (-1: HOMO)
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def Nlm_store(self) -> int:
        return self.psi_lm.shape[1]

    @property
    def Nr_store(self) -> int:
        return self.psi_lm.shape[2]


def _radial_grid(Nr, dr):
    return np.arange(Nr, dtype=np.float64) * dr


def _hartree_l0(F: np.ndarray, occ: np.ndarray, r: np.ndarray, dr: float, Nr: int) -> np.ndarray:
    """Spherical Hartree potential V_H,00(r) of the orbital density.

    rho_00(r) = sum_i occ_i sum_lambda F_{i,lambda}(r)^2 / sqrt(4 pi);
    V_00(r)  = 4 pi [ r^-1 int_0^r rho_00 r'^2 dr' + int_r^inf rho_00 r' dr' ]
    (trapezoidal cumulative integrals on the uniform grid).
    """
    rho = np.einsum("i,ilr->r", occ, F * F) / math.sqrt(4.0 * math.pi)
    rs = r[: rho.shape[0]]
    inner = np.concatenate([[0.0], np.cumsum(0.5 * dr * ((rho * rs**2)[1:] + (rho * rs**2)[:-1]))])
    g = rho * rs
    tail = np.concatenate([[0.0], np.cumsum(0.5 * dr * (g[1:] + g[:-1]))])
    outer = tail[-1] - tail
    V = np.zeros(Nr)
    with np.errstate(divide="ignore", invalid="ignore"):
        n = rho.shape[0]
        V[:n] = 4.0 * math.pi * (np.where(rs > 0, inner / np.where(rs > 0, rs, 1.0), 0.0) + outer)
        V[0] = 4.0 * math.pi * outer[0]
    # beyond the orbital support the density is zero: V = Q / r
    if n < Nr:
        Q = 4.0 * math.pi * inner[-1]
        V[n:] = Q / r[n:]
    return V


def _gram_schmidt(F: np.ndarray, r: np.ndarray, dr: float) -> np.ndarray:
    """Orthonormalise orbitals under <i|j> = int sum_lambda chi_i chi_j dr, chi = r F."""
    out = np.array(F)
    chi = out * r[None, None, : out.shape[2]]
    for i in range(out.shape[0]):
        for j in range(i):
            ov = np.sum(chi[i] * chi[j]) * dr
            out[i] -= ov * out[j]
            chi[i] -= ov * chi[j]
        nrm = math.sqrt(np.sum(chi[i] * chi[i]) * dr)
        out[i] /= nrm
        chi[i] /= nrm
    return out


def h2_like(Nr: int = 4001, dr: float = 0.01, l_cont: int = 8, seed: int = SEED_BASE + 0) -> ScanInputs:
    rng = np.random.default_rng(seed)
    l_x = min(l_cont, 10)
    Nlm = (l_cont + l_x + 1) ** 2
    r = _radial_grid(Nr, dr)
    F = np.zeros((1, Nlm, Nr))
    ls = [l for l in range(0, 9, 2)]
    c = rng.standard_normal(len(ls))
    for cl, l in zip(c, ls):
        lam = lm_to_idx(l, 0)
        if lam < Nlm:
            F[0, lam] = cl * r**l * np.exp(-1.2 * r)
    F = _gram_schmidt(F, r, dr)
    occ = np.array([2.0])
    VH = _hartree_l0(F, occ, r, dr, Nr)[None, :]
    atoms = np.array([[1.0, 0.0, 0.0, 0.7], [1.0, 0.0, 0.0, -0.7]])
    return ScanInputs("h2_like", dr, Nr, l_cont, atoms, F, np.array([-0.6]), 1, VH, seed=seed)


def _envelope_orbitals(rng, n_orb, lmax, Nlm, r, dr, zeta0=1.6, zeta_l=0.06, decay_l=4.0):
    F = np.zeros((n_orb, Nlm, r.shape[0]))
    for i in range(n_orb):
        for l in range(lmax + 1):
            amp = math.exp(-l / decay_l)
            zeta = zeta0 + zeta_l * l + 0.1 * rng.random()
            radial = r**l * np.exp(-zeta * r)
            # normalise each envelope so that amp sets its relative weight
            nrm = math.sqrt(np.sum((r * radial) ** 2) * dr)
            for m in range(-l, l + 1):
                lam = lm_to_idx(l, m)
                if lam >= Nlm:
                    continue
                F[i, lam] = amp * rng.standard_normal() * radial / nrm
    return _gram_schmidt(F, r, dr)


def h2o_like(Nr: int = 12001, dr: float = 0.005, l_cont: int = 20, lmax_orb: int = 40,
             n_orb: int = 5, seed: int = SEED_BASE + 1, Nr_store: int | None = None) -> ScanInputs:
    rng = np.random.default_rng(seed)
    l_x = min(l_cont, 10)
    Nlm = (l_cont + l_x + 1) ** 2
    lmax = min(lmax_orb, l_cont + l_x)
    rstore = Nr if Nr_store is None else min(Nr, Nr_store)
    r = _radial_grid(Nr, dr)
    F = _envelope_orbitals(rng, n_orb, lmax, Nlm, r[:rstore], dr)
    occ = np.full(n_orb, 2.0)
    VH = _hartree_l0(F, occ, r, dr, Nr)[None, :]
    R = 1.81
    half = math.radians(104.5) / 2.0
    atoms = np.array([[8.0, 0.0, 0.0, 0.0],
                      [1.0, R * math.sin(half), 0.0, R * math.cos(half)],
                      [1.0, -R * math.sin(half), 0.0, R * math.cos(half)]])
    eps = -np.sort(rng.uniform(0.4, 1.4, n_orb))[::-1]
    return ScanInputs("h2o_like", dr, Nr, l_cont, atoms, F, np.sort(eps), n_orb, VH, seed=seed)


def c8f8_like(Nr: int = 10001, dr: float = 0.01, l_cont: int = 60, lmax_orb: int = 70,
              n_orb: int = 36, seed: int = SEED_BASE + 4, Nr_store: int | None = 2500) -> ScanInputs:
    """Cubane-like C8F8 frame (C-C 1.5 A, C-F 1.33 A, 0.01 bohr jitter).

    36 doubly occupied orbitals plus one singly occupied initial-state orbital
    (the last one).  Orbital support is truncated at Nr_store points (the
    preprocessing file's Nr_orb_store), as the reference allows.
    """
    rng = np.random.default_rng(seed)
    l_x = min(l_cont, 10)
    Nlm = (l_cont + l_x + 1) ** 2
    lmax = min(lmax_orb, l_cont + l_x)
    rstore = Nr if Nr_store is None else min(Nr, Nr_store)
    r = _radial_grid(Nr, dr)
    F = _envelope_orbitals(rng, n_orb + 1, lmax, Nlm, r[:rstore], dr, zeta0=1.2, zeta_l=0.05, decay_l=6.0)
    occ = np.concatenate([np.full(n_orb, 2.0), [1.0]])
    VH = _hartree_l0(F, occ, r, dr, Nr)[None, :]
    a = 1.5 * BOHR_PER_ANGSTROM / 2.0
    cf = 1.33 * BOHR_PER_ANGSTROM
    atoms = []
    for sx in (-1, 1):
        for sy in (-1, 1):
            for sz in (-1, 1):
                p = np.array([sx, sy, sz], dtype=float) * a
                u = p / np.linalg.norm(p)
                atoms.append([6.0, *(p + 0.01 * rng.standard_normal(3))])
                atoms.append([9.0, *(p + cf * u + 0.01 * rng.standard_normal(3))])
    eps = np.sort(-rng.uniform(0.3, 1.5, n_orb + 1))
    return ScanInputs("c8f8_like", dr, Nr, l_cont, np.array(atoms), F, eps, n_orb, VH,
                      init_state=n_orb, seed=seed)


def k_grid(config: str) -> np.ndarray:
    """Momenta of the benchmark scans (k = sqrt(2E))."""
    if config == "h2_like":
        return np.arange(1, 21) * 0.1
    if config == "h2o_like":
        return np.linspace(0.05, 2.0, 200)
    raise KeyError(config)

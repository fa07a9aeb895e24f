"""The library's host-side table builders (spion-emol_b200/csrc/tables.cpp)
against the oracle, on the CPU.

These builders make every energy-independent table the kernels read: the
nuclear + Hartree multipoles V_sigma(r) (Potentials.cpp:40-88), the Gaunt
pair list of V (GauntSparse.hpp:130-180), the exchange coupling list
(WavefunctionSetup.cpp:21-81), the dipole angular tables
(DipoleMatrixElement.cpp:80-95, 628-645), the Simpson weights
(DipoleMatrixElement.cpp:142-192) and the five-point derivative (:49-74).
The GPU parity tests see them only through the final observables; here each
is compared entry by entry.  tests/host_tables_shim.cpp gives them a C
interface; it is compiled with tables.cpp and angular.cpp using the flags of
the library build.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import angular
from oracle import solver as O
from oracle.potentials import gaunt_pairs, v_sigma_table
from scatt_b200.synth import ScanInputs, lm_to_idx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "spion-emol_b200", "csrc")

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int)


def dp(a):
    return a.ctypes.data_as(D)


def ip(a):
    return a.ctypes.data_as(I)


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("tables") / "libhost_tables.so")
    cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I", CSRC,
           os.path.join(CSRC, "tables.cpp"), os.path.join(CSRC, "angular.cpp"),
           os.path.join(ROOT, "tests", "host_tables_shim.cpp"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lib = C.CDLL(out)
    lib.t_vsigma.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, D, C.c_int, D, D]
    lib.t_gaunt_pairs.argtypes = [C.c_int, C.c_int, I, I, I, I, D]
    lib.t_exchange.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, I, I, D, I]
    lib.t_dipole.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, I, I, D, D]
    lib.t_simpson.argtypes = [C.c_int, C.c_double, D]
    lib.t_five_point.argtypes = [D, C.c_int, C.c_double, D]
    return lib


def test_vsigma_table(tables):
    Nr, dr, l_cont = 301, 0.05, 4
    r = np.arange(Nr) * dr
    VH = np.zeros((4, Nr))
    VH[0] = 8.0 * np.exp(-0.3 * r)
    VH[lm_to_idx(1, 0)] = 0.7 * r * np.exp(-0.5 * r)
    atoms = np.array([[8.0, 0.0, 0.0, 0.0], [1.0, 1.43, 0.0, 1.11], [1.0, -0.7, 1.2, -0.4]])
    inp = ScanInputs(name="three_centres", dr=dr, Nr=Nr, l_cont=l_cont, atoms=atoms,
                     psi_lm=np.zeros((1, 1, Nr)), orb_energies=np.array([-0.5]), n_occ=1, V_H=VH)
    ref = v_sigma_table(inp)                                   # (n_exp, Nr)
    n_exp = ref.shape[0]
    got = np.zeros(Nr * n_exp)
    tables.t_vsigma(Nr, dr, l_cont, VH.shape[0], dp(np.ascontiguousarray(VH)), atoms.shape[0],
                    dp(np.ascontiguousarray(atoms)), dp(got))
    got = got.reshape(Nr, n_exp).T
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


@pytest.mark.parametrize("l_max", [2, 5])
def test_gaunt_pair_list(tables, l_max):
    ch = (l_max + 1) ** 2
    npair = ch * (ch + 1) // 2
    nnz = tables.t_gaunt_pairs(l_max, 0, None, None, None, None, None)
    row, col, ptr = (np.zeros(npair, np.int32), np.zeros(npair, np.int32), np.zeros(npair + 1, np.int32))
    sig, G = np.zeros(nnz, np.int32), np.zeros(nnz)
    assert tables.t_gaunt_pairs(l_max, nnz, ip(row), ip(col), ip(ptr), ip(sig), dp(G)) == nnz
    got = {}
    for p in range(npair):
        for k in range(ptr[p], ptr[p + 1]):
            got[(int(row[p]), int(col[p]), int(sig[k]))] = G[k]
    pairs, Gs = gaunt_pairs(l_max)
    Gs = Gs.tocsr()
    ref = {}
    for i, (mp, mu) in enumerate(pairs):
        for k in range(Gs.indptr[i], Gs.indptr[i + 1]):
            ref[(int(mp), int(mu), int(Gs.indices[k]))] = Gs.data[k]
    assert got.keys() == ref.keys()
    assert max(abs(got[k] - ref[k]) for k in ref) <= 1e-15


@pytest.mark.parametrize("n_mu,n_sigma,n_lambda", [(9, 9, 25), (25, 16, 64)])
def test_exchange_list(tables, n_mu, n_sigma, n_lambda):
    nnz = tables.t_exchange(n_mu, n_sigma, n_lambda, 0, None, None, None, None)
    ptr, lam, G = np.zeros(n_mu * n_sigma + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    nlm = C.c_int(0)
    assert tables.t_exchange(n_mu, n_sigma, n_lambda, nnz, ip(ptr), ip(lam), dp(G), C.byref(nlm)) == nnz
    got = {}
    for row in range(n_mu * n_sigma):
        mu, s = divmod(row, n_sigma)
        for k in range(ptr[row], ptr[row + 1]):
            got[(mu, int(lam[k]), s)] = G[k]
    ref = {(mu, la, si): v for mu, la, si, v in angular.build_G_vector(n_mu, n_lambda, n_sigma)}
    assert got.keys() == ref.keys()
    assert max(abs(got[k] - ref[k]) for k in ref) <= 1e-15
    assert nlm.value == max(la for _, la, _ in ref) + 1


def test_dipole_tables(tables):
    n_mu, n_lambda = 36, 64
    for qi, q in enumerate((1, -1, 0)):                       # x, y, z
        nnz = tables.t_dipole(n_mu, n_lambda, qi, 0, None, None, None, None)
        ptr, nu = np.zeros(n_mu + 1, np.int32), np.zeros(nnz, np.int32)
        a, c = np.zeros(nnz), np.zeros(nnz)
        assert tables.t_dipole(n_mu, n_lambda, qi, nnz, ip(ptr), ip(nu), dp(a), dp(c)) == nnz
        dense_a = np.zeros((n_mu, n_lambda))
        dense_c = np.zeros((n_mu, n_lambda))
        for mu in range(n_mu):
            for k in range(ptr[mu], ptr[mu + 1]):
                dense_a[mu, nu[k]] = a[k]
                dense_c[mu, nu[k]] = c[k]
        ref_a = np.zeros((n_mu, n_lambda))
        for mu in range(n_mu):
            lmu, mmu = angular.idx_to_lm(mu)
            for v in range(n_lambda):
                lnu, mnu = angular.idx_to_lm(v)
                if abs(lmu - lnu) == 1:
                    ref_a[mu, v] = angular.angular_dipole(lmu, mmu, q, lnu, mnu)
                    if dense_a[mu, v] != 0.0:
                        assert dense_c[mu, v] == angular.velocity_coef(lmu, lnu)
        assert np.max(np.abs(dense_a - ref_a)) <= 1e-15


def test_simpson_weights(tables):
    rng = np.random.default_rng(3)
    h = 0.01
    for n in range(0, 40):
        w = np.zeros(max(n, 1))
        tables.t_simpson(n, h, dp(w))
        f = rng.standard_normal(n)
        want = O.simpson(f, h)
        got = float(np.dot(w[:n], f)) if n else 0.0
        assert abs(got - want) <= 1e-14 * max(1.0, np.sum(np.abs(f)) * h)
    # n = 4: the 1/3 rule over one point counts f[0] twice before the 3/8 rule
    w = np.zeros(4)
    tables.t_simpson(4, h, dp(w))
    assert w[0] == pytest.approx(2.0 * h / 3.0 + 3.0 * h / 8.0, rel=1e-15)


def test_five_point_derivative(tables):
    rng = np.random.default_rng(4)
    for n in range(1, 30):
        f = rng.standard_normal(n)
        got = np.zeros(n)
        tables.t_five_point(dp(f), n, 0.02, dp(got))
        assert np.array_equal(got, O.five_point_derivative(f, 0.02))

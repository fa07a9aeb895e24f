"""The C++ host interface (spion-emol_b200/host/scatt_b200.hpp) through its
command-line driver: solve and inverse modes against the oracle and numpy,
and the reference's error behaviour (a thrown std::runtime_error carrying the
library's message; here the driver's exit status 2)."""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "spion-emol_b200")
DRIVER = os.path.join(PKG, "host", "scan_driver")

from scatt_b200 import _lib, synth  # noqa: E402


def _driver():
    if not os.path.exists(DRIVER):
        sys.path.insert(0, PKG)
        import build as _b
        _b.build()
    return DRIVER


def _has_gpu():
    try:
        return _lib.device_count() > 0
    except Exception:
        return False


def write_inputs(path, inp, Es, allow_closed=True):
    psi = np.ascontiguousarray(inp.psi_lm, dtype="<f8")
    vh = np.ascontiguousarray(inp.V_H, dtype="<f8")
    at = np.ascontiguousarray(inp.atoms, dtype="<f8")
    E = np.ascontiguousarray(Es, dtype="<f8")
    hdr = [inp.Nr, inp.l_cont, inp.n_occ, psi.shape[0], psi.shape[1], psi.shape[2], inp.init_state,
           vh.shape[0], at.shape[0], inp.pol_form, 0, E.size, 1 if allow_closed else 0]
    with open(path, "wb") as f:
        f.write(struct.pack("<13i", *hdr))
        f.write(struct.pack("<4d", inp.dr, inp.alpha_pol, inp.r_c, 1e-15))
        for a in (psi, vh, at, E):
            f.write(a.tobytes())


def read_results(path, nE):
    raw = open(path, "rb").read()
    Np = struct.unpack_from("<i", raw, 0)[0]
    vals = np.frombuffer(raw, dtype="<f8", offset=4)
    per = 1 + 3 * Np * Np + 12 * Np + 6
    out = []
    for e in range(nE):
        v = vals[e * per:(e + 1) * per]
        o = 1
        K = v[o:o + Np * Np].reshape(Np, Np, order="F"); o += Np * Np
        A = v[o:o + Np * Np].reshape(Np, Np, order="F"); o += Np * Np
        B = v[o:o + Np * Np].reshape(Np, Np, order="F"); o += Np * Np
        D = []
        for s in range(6):
            D.append(v[o:o + Np] + 1j * v[o + Np:o + 2 * Np]); o += 2 * Np
        sig = v[o:o + 6]
        out.append(dict(status=int(v[0]), K=K, A=A, B=B, D=np.array(D), sigma=sig))
    return Np, out


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_driver_reports_missing_device(tmp_path):
    inp = synth.h2_like(Nr=201, dr=0.05, l_cont=1)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    write_inputs(fin, inp, [0.5])
    r = subprocess.run([_driver(), "solve", str(fin), str(fout)], capture_output=True, text=True)
    assert r.returncode == 2
    assert "no CUDA device" in r.stderr
    r = subprocess.run([_driver(), "stepper", "8"], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stderr
    m = tmp_path / "m.bin"
    m.write_bytes(struct.pack("<i", 2) + np.eye(2).tobytes())
    r = subprocess.run([_driver(), "inverse", str(m), str(tmp_path / "x.bin")], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stderr


@pytest.mark.gpu
def test_driver_solve_matches_oracle(tmp_path):
    from oracle import solver as O
    inp = synth.h2_like(Nr=801, dr=0.05, l_cont=2)
    Es = [0.5, 1.2]
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    write_inputs(fin, inp, Es)
    r = subprocess.run([_driver(), "solve", str(fin), str(fout)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    Np, res = read_results(fout, len(Es))
    st = O.make_setup(inp)
    assert Np == st.n_mu
    for E, g in zip(Es, res):
        ref = O.solve_energy(st, E)
        assert g["status"] == 0
        assert np.max(np.abs(g["K"] - ref.K_kme)) <= 1e-9 * np.max(np.abs(ref.K_kme))
        for s in range(6):
            Dr = ref.slices[s]["D"]
            assert np.max(np.abs(g["D"][s] - Dr)) <= 1e-9 * max(np.max(np.abs(Dr)), 1e-300)


@pytest.mark.gpu
def test_driver_inverse_and_singular_throw(tmp_path):
    rng = np.random.default_rng(11)
    n = 50
    A = rng.standard_normal((n, n)) + 6.0 * np.eye(n)
    m, x = tmp_path / "m.bin", tmp_path / "x.bin"
    m.write_bytes(struct.pack("<i", n) + np.asfortranarray(A).tobytes(order="F"))
    r = subprocess.run([_driver(), "inverse", str(m), str(x)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    X = np.frombuffer(x.read_bytes(), dtype="<f8").reshape(n, n, order="F")
    assert np.max(np.abs(X - np.linalg.inv(A))) <= 1e-12 * np.max(np.abs(np.linalg.inv(A)))
    m.write_bytes(struct.pack("<i", 3) + np.ones((3, 3)).tobytes())
    r = subprocess.run([_driver(), "inverse", str(m), str(x)], capture_output=True, text=True)
    assert r.returncode == 2 and "singular" in r.stderr


@pytest.mark.gpu
def test_driver_seam_classes():
    # built as the reference's stage classes build them (GpuContext, then the
    # stepper): W_inv = I/2, R_prev_inv = 0 gives Rinv = (6 I - 10 I)^-1 = -I/4,
    # and the dipole engine's V . (2 I) = 2 V on small integers; both exact in
    # binary floating point (the driver exits 3 otherwise)
    r = subprocess.run([_driver(), "stepper", "8"], capture_output=True, text=True)
    assert r.returncode == 0, (r.stdout, r.stderr)
    err_fwd, err_dip = (float(x) for x in r.stdout.split())
    assert err_fwd < 1e-15 and err_dip == 0.0


def test_seam_headers_take_the_reference_calls(tmp_path):
    """tests/host_seam_check.cpp makes the reference's stage-class calls into
    the device seam, as written there, against host/seam/scatt/*.hpp: it must
    compile warning-free and, without a GPU, show the no-device behaviour."""
    _driver()                                        # the library is built
    exe = tmp_path / "seam_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"),
           "-I", os.path.join(PKG, "host", "seam"), os.path.join(ROOT, "tests", "host_seam_check.cpp"),
           "-L", PKG, "-lscatt_b200", f"-Wl,-rpath,{PKG}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.stdout, r.stderr)


def test_psi_and_cc_dipole_calls_compile(tmp_path):
    """tests/host_psi_check.cpp calls ScanSolver::psi, psi_into and
    compute_cc_dipole of the C++ interface: warning-free, and without a GPU
    each throws the library's no-device error."""
    _driver()
    exe = tmp_path / "psi_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"),
           os.path.join(ROOT, "tests", "host_psi_check.cpp"),
           "-L", PKG, "-lscatt_b200", f"-Wl,-rpath,{PKG}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)


def test_preprocessing_interface_compiles_and_reads_molden(tmp_path):
    """tests/host_preproc_check.cpp uses host/scatt_preproc.hpp as the
    reference's preprocessing driver would: warning-free; the Molden reader
    runs on the host; the device steps report a missing device."""
    _driver()
    exe = tmp_path / "preproc_check"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"),
           os.path.join(ROOT, "tests", "host_preproc_check.cpp"),
           "-L", PKG, "-lscatt_b200", f"-Wl,-rpath,{PKG}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)

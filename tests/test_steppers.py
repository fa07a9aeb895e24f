"""The per-radial-step compatibility seam (GpuForwardStepper, GpuSinvStepper,
GpuBackStepper of src/scatt/GpuPropagate.hpp) against numpy, as the
reference's src/tests/test_gpu_steppers.cpp checks its own steppers:
a single forward step and a chain of steps (1e-11 relative), the back step
(Z <- Rinv Z, Y = W_inv Z split into psi and f) and the Schur inverse."""
import ctypes as C

import numpy as np
import pytest

from scatt_b200 import _lib

vp = C.c_void_p
dp = C.POINTER(C.c_double)


def _bind():
    L = _lib.lib()
    L.scatt_fwd_stepper_create.argtypes = [C.c_int, C.c_int, C.POINTER(vp)]
    L.scatt_fwd_stepper_destroy.argtypes = [vp]
    L.scatt_fwd_stepper_init.argtypes = [vp, dp]
    L.scatt_fwd_stepper_step.argtypes = [vp, dp, dp, dp]
    L.scatt_sinv_stepper_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    L.scatt_sinv_stepper_destroy.argtypes = [vp]
    L.scatt_sinv_stepper_step.argtypes = [vp, dp, dp, dp, dp, dp]
    L.scatt_back_stepper_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    L.scatt_back_stepper_destroy.argtypes = [vp]
    L.scatt_back_stepper_init.argtypes = [vp, dp]
    L.scatt_back_stepper_step.argtypes = [vp, dp, dp, dp, dp]
    L.scatt_back_stepper_get_z.argtypes = [vp, dp]
    return L


def F(a):
    return np.asfortranarray(a, dtype=np.float64)


def P(a):
    return a.ctypes.data_as(dp)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def sym_rand(rng, n, scale):
    M = rng.standard_normal((n, n))
    return scale * 0.5 * (M + M.T)


def test_no_device_is_reported():
    if _lib.device_count() > 0:
        pytest.skip("checks the no-device error path")
    L = _bind()
    h = vp()
    assert L.scatt_fwd_stepper_create(0, 8, C.byref(h)) == 7
    assert L.scatt_sinv_stepper_create(0, 8, 4, C.byref(h)) == 7
    assert L.scatt_back_stepper_create(0, 8, 4, C.byref(h)) == 7


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 700])
def test_forward_step_and_chain(n):
    L = _bind()
    rng = np.random.default_rng(42)
    Rprev = F(sym_rand(rng, n, 0.1 / np.sqrt(n)))
    Ws = [F(0.9 * np.eye(n) + sym_rand(rng, n, 0.01 / np.sqrt(n))) for _ in range(5)]
    h = vp()
    _lib.check(L.scatt_fwd_stepper_create(0, n, C.byref(h)))
    try:
        _lib.check(L.scatt_fwd_stepper_init(h, P(Rprev)))
        expect = Rprev.copy()
        for W in Ws:
            M = np.linalg.inv(12.0 * W - 10.0 * np.eye(n) - expect)
            expect = 0.5 * (M + M.T)
            out = F(np.zeros((n, n)))
            asym = C.c_double(-1.0)
            _lib.check(L.scatt_fwd_stepper_step(h, P(W), P(out), C.byref(asym)))
            assert rel(out, expect) < 1e-11
            assert asym.value == 0.0
    finally:
        L.scatt_fwd_stepper_destroy(h)


@pytest.mark.gpu
def test_forward_step_reports_a_singular_matrix():
    L = _bind()
    n = 16
    h = vp()
    _lib.check(L.scatt_fwd_stepper_create(0, n, C.byref(h)))
    try:
        # 12 W - 10 I - Rprev = 6 - 10 + 4 = 0 exactly for W = I / 2, Rprev = -4 I
        _lib.check(L.scatt_fwd_stepper_init(h, P(F(-4.0 * np.eye(n)))))
        W = F(0.5 * np.eye(n))
        out = F(np.zeros((n, n)))
        assert L.scatt_fwd_stepper_step(h, P(W), P(out), None) == 4        # SCATT_ERR_SINGULAR
        assert b"GpuForwardStepper" in _lib.lib().scatt_last_error()
    finally:
        L.scatt_fwd_stepper_destroy(h)


@pytest.mark.gpu
@pytest.mark.parametrize("npsi,nf", [(48, 30), (441, 121)])
def test_sinv_step(npsi, nf):
    L = _bind()
    rng = np.random.default_rng(43)
    A = F(np.eye(npsi) * 1.2 + sym_rand(rng, npsi, 0.02 / np.sqrt(npsi)))
    B = F(0.05 * rng.standard_normal((npsi, nf)) / np.sqrt(nf))
    d = np.ascontiguousarray(rng.uniform(0.5, 1.5, nf))
    h = vp()
    _lib.check(L.scatt_sinv_stepper_create(0, npsi, nf, C.byref(h)))
    try:
        out = F(np.zeros((npsi, npsi)))
        _lib.check(L.scatt_sinv_stepper_step(h, P(A), P(B), P(d), P(out), None))
        M = np.linalg.inv(A - (B * d[None, :]) @ B.T)
        assert rel(out, 0.5 * (M + M.T)) < 1e-11
        _lib.check(L.scatt_sinv_stepper_step(h, P(A), None, None, P(out), None))     # inverse only
        M = np.linalg.inv(A)
        assert rel(out, 0.5 * (M + M.T)) < 1e-11
    finally:
        L.scatt_sinv_stepper_destroy(h)


@pytest.mark.gpu
@pytest.mark.parametrize("nt,npsi", [(40, 25), (600, 441)])
def test_back_steps(nt, npsi):
    L = _bind()
    rng = np.random.default_rng(44)
    nf = nt - npsi
    Z = F(rng.standard_normal((nt, npsi)))
    h = vp()
    _lib.check(L.scatt_back_stepper_create(0, nt, npsi, C.byref(h)))
    try:
        _lib.check(L.scatt_back_stepper_init(h, P(Z)))
        z = Z.copy()
        for k in range(3):
            R = F(rng.standard_normal((nt, nt)) / np.sqrt(nt))
            W = F(rng.standard_normal((nt, nt)) / np.sqrt(nt))
            psi = F(np.zeros((npsi, npsi)))
            f = F(np.zeros((nf, npsi)))
            _lib.check(L.scatt_back_stepper_step(h, P(R), P(W), P(psi), P(f) if k != 1 else None))
            z = R @ z
            Y = W @ z
            assert rel(psi, Y[:npsi]) < 1e-12
            if k != 1:
                assert rel(f, Y[npsi:]) < 1e-12
        zg = F(np.zeros((nt, npsi)))
        _lib.check(L.scatt_back_stepper_get_z(h, P(zg)))
        assert rel(zg, z) < 1e-12
    finally:
        L.scatt_back_stepper_destroy(h)

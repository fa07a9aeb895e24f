"""scatt_inverse_batched_noalloc against the allocating scatt_inverse_batched.

The allocation-free entry point is for callers that cannot call cudaMalloc
(their own allocator owns the device's free memory, or they cannot take the
synchronisation of cudaMalloc / cudaFree); it uses one static device scratch
array instead.  Checked here: the same inverses on two calls in a row (the
array keeps the previous call's contents), singular-pivot reporting, and the
size limits.  The file is collected last so it also runs after every other
GPU test."""
import numpy as np
import pytest

from scatt_b200 import _lib

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_matches_allocating_inverse_two_calls():
    rng = np.random.default_rng(2026)
    A1 = rng.standard_normal((3, 200, 200)) + 4.0 * np.eye(200)
    M = rng.standard_normal((5, 77, 77))
    A2 = M + np.transpose(M, (0, 2, 1)) + 20.0 * np.eye(77)
    for A, sym in ((A1, False), (A2, True)):
        ref, st_ref = _lib.inverse_batched(A, symmetrize=sym)
        got, st = _lib.inverse_batched(A, symmetrize=sym, noalloc=True)
        assert np.all(st == 0) and np.all(st_ref == 0)
        for b in range(A.shape[0]):
            assert _rel(got[b], ref[b]) < 1e-13
            assert np.max(np.abs(got[b] @ A[b] - np.eye(A.shape[1]))) < 1e-10


@pytest.mark.parametrize("n,count,scheme", [(1046, 2, 0), (200, 3, 3)])
def test_noalloc_row_contiguous_scheme_two_calls(n, count, scheme):
    """Orders above 512 (or scheme 3 forced) run the row-contiguous inverse
    without look-ahead, over several 64-column windows; order 1046 with two
    matrices needs about 55 MB of the 64 MiB array."""
    rng = np.random.default_rng(n)
    M = rng.standard_normal((count, n, n))
    A = M + np.transpose(M, (0, 2, 1)) + 2.0 * np.sqrt(n) * np.eye(n)
    _lib.set_inverse_blocking(scheme)
    try:
        ref, st_ref = _lib.inverse_batched(A, symmetrize=True)
        for _ in range(2):
            got, st = _lib.inverse_batched(A, symmetrize=True, noalloc=True)
            assert np.all(st == 0) and np.all(st_ref == 0)
            for b in range(count):
                assert _rel(got[b], ref[b]) < 1e-12
                assert np.max(np.abs(got[b] @ A[b] - np.eye(n))) < 1e-9
    finally:
        _lib.set_inverse_blocking(0)


def test_noalloc_reports_singular_like_allocating():
    A = np.ones((2, 6, 6))
    code = _lib.lib().scatt_inverse_batched_noalloc
    st = np.zeros((2, 2), dtype=np.int32)
    out = np.empty_like(A)
    rc = code(6, 2, _lib.as_dptr(np.ascontiguousarray(A)), _lib.as_dptr(out), 0, _lib.as_iptr(st))
    assert rc == 4                                   # SCATT_ERR_SINGULAR
    assert np.all(st[:, 0] == 1)


@pytest.mark.parametrize("n,count", [(1281, 1), (1000, 16), (8, 257)])
def test_noalloc_rejects_oversized(n, count):
    rc = _lib.lib().scatt_inverse_batched_noalloc(n, count, _lib.as_dptr(np.zeros(1)),
                                                  _lib.as_dptr(np.zeros(1)), 0, None)
    assert rc == 3                                   # SCATT_ERR_SIZE, before any device work

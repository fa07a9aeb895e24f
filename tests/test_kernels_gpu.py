"""Device building blocks against numpy fp64: batched GJ inverse and DMMA GEMM."""
import numpy as np
import pytest

from scatt_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,count", [(1, 1), (5, 3), (16, 2), (17, 2), (40, 4), (64, 1), (100, 3), (162, 2), (257, 1), (441, 1), (1046, 1)])
def test_inverse_matches_numpy(n, count):
    rng = np.random.default_rng(42 + n)
    A = rng.standard_normal((count, n, n)) + 3.0 * np.eye(n)
    inv, st = _lib.inverse_batched(A)
    assert np.all(st == 0)
    for b in range(count):
        ref = np.linalg.inv(A[b])
        err = np.max(np.abs(inv[b] - ref)) / np.max(np.abs(ref))
        assert err < 1e-12, (n, b, err)


def test_inverse_needs_pivoting():
    # zero diagonal: no-pivot elimination would fail immediately
    rng = np.random.default_rng(7)
    n = 48
    P = np.eye(n)[rng.permutation(n)]
    A = P @ (np.diag(rng.uniform(1, 2, n)) + 0.1 * rng.standard_normal((n, n)))
    A[np.diag_indices(n)] = 0.0
    inv, st = _lib.inverse_batched(A)
    assert np.all(st == 0)
    assert np.max(np.abs(inv @ A - np.eye(n))) < 1e-11


def test_inverse_symmetrized():
    rng = np.random.default_rng(3)
    n = 130
    M = rng.standard_normal((n, n))
    S = M + M.T + n * np.eye(n)
    inv, st = _lib.inverse_batched(S, symmetrize=True)
    assert np.array_equal(inv, inv.T)
    ref = np.linalg.inv(S)
    assert np.max(np.abs(inv - ref)) / np.max(np.abs(ref)) < 1e-13


def test_inverse_singular_reports_status():
    A = np.ones((3, 4, 4))
    inv, st = _lib.inverse_batched(A)
    assert np.all(st[:, 0] == 1)


@pytest.mark.parametrize("opA,opB", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (7, 13, 5), (11, 1046, 1046), (16, 130, 77), (17, 70, 33), (64, 64, 16),
                                   (65, 63, 17), (128, 64, 32), (129, 65, 33), (256, 192, 96), (200, 130, 441),
                                   (441, 605, 441)])
def test_dgemm_matches_numpy(opA, opB, M, N, K):
    rng = np.random.default_rng(M * 1000 + N + K)
    A = rng.standard_normal((K, M) if opA else (M, K))
    B = rng.standard_normal((N, K) if opB else (K, N))
    C0 = rng.standard_normal((M, N))
    out = _lib.dgemm(A, B, C0, alpha=-0.75, beta=0.5, opA=opA, opB=opB)
    ref = -0.75 * ((A.T if opA else A) @ (B.T if opB else B)) + 0.5 * C0
    assert np.max(np.abs(out - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref))) * np.sqrt(K + 1)


@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("n", [77, 441, 600, 1046])
def test_inverse_every_scheme(scheme, n):
    """Single-level, column-major two-level and row-contiguous two-level
    inverses (64- and 128-column windows, single-CTA and small cluster
    panels) against numpy; odd orders take the 8-byte copy paths."""
    rng = np.random.default_rng(1000 + n)
    A = rng.standard_normal((2, n, n)) + 4.0 * np.sqrt(n) * np.eye(n)
    try:
        _lib.set_inverse_blocking(scheme)
        inv, st = _lib.inverse_batched(A, symmetrize=False)
    finally:
        _lib.set_inverse_blocking(0)
    assert np.all(st == 0)
    for b in range(2):
        ref = np.linalg.inv(A[b])
        assert np.max(np.abs(inv[b] - ref)) / np.max(np.abs(ref)) < 1e-12


@pytest.mark.parametrize("n,count", [(300, 4), (700, 3)])
def test_autotuned_inverse_is_kept_and_exact(n, count):
    """The autotuner keeps a valid configuration for (order, batch); inverses
    of exactly that order and batch then run it and still equal numpy's."""
    t = _lib.autotune_inverse(n, count, reps=1)
    assert t["scheme"] in (2, 3) and 0 <= t["panel"] <= 6 and t["look_ahead"] in (0, 1) and t["ms"] > 0
    assert t["window"] == 64 or (t["scheme"] == 3 and t["window"] == 128)
    assert t["panel"] == 6 or n <= (256, 512, 768, 1152, 1280)[t["panel"]]
    rng = np.random.default_rng(n + count)
    M = rng.standard_normal((count, n, n))
    A = M + np.transpose(M, (0, 2, 1)) + 2.0 * np.sqrt(n) * np.eye(n)
    got, st = _lib.inverse_batched(A, symmetrize=True)
    assert np.all(st == 0)
    for b in range(count):
        ref = np.linalg.inv(A[b])
        assert np.max(np.abs(got[b] - ref)) / np.max(np.abs(ref)) < 1e-12


@pytest.mark.parametrize("n,scheme", [(1281, 0), (1281, 4), (2048, 0), (2048, 4), (5306, 0), (5306, 4)])
def test_inverse_cluster_panel_orders(n, scheme):
    """Orders above one CTA's panel run the cluster panel (CTAs of one
    thread-block cluster share the pivot search through distributed shared
    memory), with 64- (scheme 0 picks scheme 3) and 128-column windows; a
    symmetric and a general batch against numpy."""
    rng = np.random.default_rng(5000 + n)
    M = rng.standard_normal((2, n, n))
    A = M + np.transpose(M, (0, 2, 1)) + 4.0 * np.sqrt(n) * np.eye(n)
    try:
        _lib.set_inverse_blocking(scheme)
        _cluster_checks(rng, n, A)
    finally:
        _lib.set_inverse_blocking(0)


def _cluster_checks(rng, n, A):
    got, st = _lib.inverse_batched(A, symmetrize=True)
    assert np.all(st == 0)
    assert np.array_equal(got[0], got[0].T)
    for b in range(2):
        ref = np.linalg.inv(A[b])
        assert np.max(np.abs(got[b] - ref)) / np.max(np.abs(ref)) < 1e-12, (n, b)
    if n <= 2048:
        G = rng.standard_normal((1, n, n)) + 4.0 * np.sqrt(n) * np.eye(n)
        got, st = _lib.inverse_batched(G, symmetrize=False)
        assert np.all(st == 0)
        ref = np.linalg.inv(G[0])
        assert np.max(np.abs(got[0] - ref)) / np.max(np.abs(ref)) < 1e-12


def test_inverse_cluster_panel_pivots_across_ctas():
    """Zero diagonal under a random row permutation: every pivot sits in a
    row owned by some other CTA of the cluster than the column's own."""
    rng = np.random.default_rng(77)
    n = 2500
    P = np.eye(n)[rng.permutation(n)]
    A = P @ (np.diag(rng.uniform(1, 2, n)) + 0.01 * rng.standard_normal((n, n)))
    A[np.diag_indices(n)] = 0.0
    got, st = _lib.inverse_batched(A[None], symmetrize=False)
    assert np.all(st == 0)
    assert np.max(np.abs(got[0] @ A - np.eye(n))) < 1e-10


def test_inverse_cluster_panel_singular_status():
    inv, st = _lib.inverse_batched(np.ones((2, 1500, 1500)))
    assert np.all(st[:, 0] == 1)
    assert np.all(st[:, 1] == 1)

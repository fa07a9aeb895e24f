"""The C-ABI library loads on a CPU host and exports every declared symbol."""
import ctypes
import os
import re

import numpy as np

from scatt_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "scatt_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|double|void|char)\s*\**\s*(scatt_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("scatt_ctx_create", "scatt_upload_static", "scatt_solve_batch", "scatt_inverse_batched",
              "scatt_dgemm", "scatt_gaunt_real", "scatt_riccati_j"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_device_count_without_gpu():
    assert b"sm_100a" in _lib.lib().scatt_version()
    assert _lib.device_count() >= 0


def test_compute_entry_points_fail_loudly_without_device():
    if _lib.device_count() > 0:
        return
    A = np.eye(3)[None]
    code = _lib.lib().scatt_inverse_batched(3, 1, _lib.as_dptr(np.ascontiguousarray(A)),
                                            _lib.as_dptr(np.zeros_like(A)), 0, None)
    assert code == 7          # SCATT_ERR_NO_DEVICE: no CPU fallback
    assert b"no CUDA device" in _lib.lib().scatt_last_error()


def test_every_compute_entry_point_reports_no_device():
    """Without a CUDA device every compute entry point returns
    SCATT_ERR_NO_DEVICE (7) with the library's message: there is no CPU
    path behind any of them."""
    if _lib.device_count() > 0:
        return
    L = _lib.lib()
    A = np.ascontiguousarray(np.eye(4)[None])
    out = np.zeros_like(A)
    C = np.zeros((4, 4))
    ms = np.zeros(1)
    calls = {
        "scatt_inverse_batched": lambda: L.scatt_inverse_batched(4, 1, _lib.as_dptr(A), _lib.as_dptr(out), 0, None),
        "scatt_inverse_batched_noalloc": lambda: L.scatt_inverse_batched_noalloc(
            4, 1, _lib.as_dptr(A), _lib.as_dptr(out), 0, None),
        "scatt_dgemm": lambda: L.scatt_dgemm(0, 0, 4, 4, 4, 1.0, _lib.as_dptr(C), 4, _lib.as_dptr(C), 4, 0.0,
                                             _lib.as_dptr(C), 4),
        "scatt_bench_inverse": lambda: L.scatt_bench_inverse(8, 1, 1, _lib.as_dptr(ms)),
        "scatt_ctx_create": lambda: L.scatt_ctx_create(0, ctypes.byref(ctypes.c_void_p())),
        "scatt_hartree": lambda: L.scatt_hartree(1, 4, 8, 0.0, 0.1, _lib.as_dptr(np.ones((4, 8))),
                                                 _lib.as_dptr(np.zeros((4, 8)))),
        "scatt_sce_project": lambda: L.scatt_sce_project(1, 2, 0, _lib.as_dptr(np.ones((2, 2, 4))),
                                                         _lib.as_dptr(np.zeros((4, 2)))),
        "scatt_cc_dipole": lambda: L.scatt_cc_dipole(4, 4, 6, 0, 0.1, 0, _lib.as_dptr(np.ones((6, 4, 4))), 1,
                                                     _lib.as_dptr(np.ones((6, 4, 4))), _lib.as_dptr(np.zeros((4, 4)))),
        "scatt_sce_basis": lambda: L.scatt_sce_basis(
            1, 2, 0.0, 0.1, _lib.as_dptr(np.zeros(3)), 1, _lib.as_iptr(np.zeros(1, dtype=np.int32)),
            _lib.as_iptr(np.ones(1, dtype=np.int32)), _lib.as_dptr(np.zeros(3)), _lib.as_dptr(np.ones(1)),
            _lib.as_dptr(np.ones(1)), 1, _lib.as_dptr(np.ones((1, 1))), _lib.as_dptr(np.ones(1)), 0, 0,
            _lib.as_dptr(np.zeros((1, 4, 2))), _lib.as_dptr(np.zeros((4, 2))), None),
    }
    for name, call in calls.items():
        assert call() == 7, name
        assert b"no CUDA device" in L.scatt_last_error(), name


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """The package has no fallback when the built library is absent: the
    first use raises with the build instruction."""
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libscatt_b200.so"))
    try:
        _lib.lib()
    except _lib.ScattError as e:
        assert "is missing" in str(e) and "build.py" in str(e)
    else:
        raise AssertionError("lib() returned without the library")

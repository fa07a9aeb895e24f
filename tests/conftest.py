import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_PY = os.path.join(ROOT, "spion-emol_b200", "python")
for p in (ROOT, PKG_PY):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


def _has_gpu():
    try:
        from scatt_b200 import _lib
        return _lib.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def pytest_sessionfinish(session, exitstatus):
    """Release what the tests left for the garbage collector (solvers, scans
    and adjoints in reference cycles hold device memory and library handles)
    while the CUDA runtime and torch are still fully alive, instead of at
    interpreter shutdown, and let the device finish its queued work."""
    import gc
    gc.collect()
    if "torch" in sys.modules:
        torch = sys.modules["torch"]
        if torch.cuda.is_available() and torch.cuda.is_initialized():
            torch.cuda.synchronize()

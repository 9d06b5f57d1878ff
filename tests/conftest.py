"""Shared pytest setup: the ``gpu`` marker, repo paths and device detection."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


_HAS_GPU = None


def has_gpu() -> bool:
    """True when the CUDA library can create a solver on a device."""
    global _HAS_GPU
    if _HAS_GPU is None:
        import basements_b200 as bm
        h = __import__("ctypes").c_void_p()
        st = bm.lib().bm_solver_create(0.1, None, __import__("ctypes").byref(h))
        if st == 0:
            bm.lib().bm_solver_destroy(h)
        _HAS_GPU = st == 0
    return _HAS_GPU


def pytest_collection_modifyitems(config, items):
    for item in items:
        if "gpu" in item.keywords:
            try:
                ok = has_gpu()
            except ImportError:
                ok = True  # let the test fail loudly: the CUDA library is missing
            if not ok:
                item.add_marker(pytest.mark.skip(reason="no CUDA device visible"))

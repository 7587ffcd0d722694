import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


def pytest_collection_modifyitems(config, items):
    """GPU tests fail loudly when the library or the device is missing on a
    GPU run; on a CPU-only host (no device) they are skipped."""
    try:
        from qublar_b200 import device_count
        n = device_count()
    except Exception:
        n = 0
    if n > 0:
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)

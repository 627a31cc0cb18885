import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "classical-quantum-sim-optimizer_b200"
for p in (str(ROOT), str(PKG), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def pytest_collection_modifyitems(config, items):
    # GPU tests are skipped automatically when no CUDA device is visible, so a
    # plain `pytest tests/` on a CPU-only machine still passes.
    has_gpu = False
    try:
        import ctypes

        cuda = ctypes.CDLL("libcuda.so.1")
        count = ctypes.c_int(0)
        has_gpu = cuda.cuInit(0) == 0 and cuda.cuDeviceGetCount(ctypes.byref(count)) == 0 and count.value > 0
    except OSError:
        has_gpu = False
    if has_gpu or os.environ.get("DQSIM_FORCE_GPU_TESTS"):
        return
    skip = pytest.mark.skip(reason="no CUDA device visible")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)

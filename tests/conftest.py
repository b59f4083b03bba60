"""pytest configuration: the gpu marker and the native builds.

CPU runs (-m "not gpu") build the oracle and the CUDA library in-tree if
they are missing (nvcc cross-compiles without a GPU); GPU tests call the
library through its C ABI.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    oracle_so = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       capture_output=True)
    lib_so = os.path.join(ROOT, "wloop_b200", "_lib", "libwloop_b200.so")
    if not os.path.exists(lib_so):
        subprocess.run([sys.executable, os.path.join(ROOT, "wloop_b200", "build.py")], check=True,
                       capture_output=True)


def _has_gpu():
    try:
        import wloop_b200
        return wloop_b200.device_count() > 0
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)

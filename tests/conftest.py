"""Test configuration.

Markers: tests that need a GPU carry ``@pytest.mark.gpu``; everything else runs
on a CPU-only machine.  The CPU oracle (oracle/) is the checker for every
parity test; the CUDA library is driven through its C ABI (libifc.so) via the
ctypes binding in incompflow-cuda_b200/python/ifc.py.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "incompflow-cuda_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libifc.so")


def _ensure_built():
    lib = os.path.join(ROOT, "incompflow-cuda_b200", "lib", "libifc.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "incompflow-cuda_b200"), "lib"], check=True)
    import oracle  # noqa: E402

    oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def gpu_ok():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True

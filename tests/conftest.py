"""Shared test setup.

Markers:
  gpu -- needs a CUDA device (B200); run with ``pytest -m gpu``.

The CPU-only suite (``-m "not gpu"``) covers the oracle against the reference's
golden vectors, the host-side logic, and that the C-ABI library loads and
exports what include/mela.h declares.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device")


def _ensure_built():
    # The checker and the library are built in place when missing (this
    # container); on a machine without the reference tree the prebuilt
    # oracle/_ref objects are used as they are.
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       capture_output=True)
    lib = os.path.join(ROOT, "mex_linear_algebra_b200", "libmela_b200.so")
    if not os.path.exists(lib):
        from mex_linear_algebra_b200 import build
        build.build()


_ensure_built()


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")

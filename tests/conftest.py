"""Shared test setup: import paths, the gpu marker, and builds on demand."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "ni-cr_oxidation_phase-field_simulation_b200"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # The CUDA library and the oracle are built in-tree; build them if absent
    # (nvcc cross-compiles without a GPU).
    if not (PKG / "lib" / "libnicr.so").exists():
        subprocess.run(["make", "-C", str(PKG), "-j8"], check=True, capture_output=True)
    if not (ROOT / "oracle" / "_build" / "libnicr_oracle.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True, capture_output=True)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.fail("this test needs a CUDA device")

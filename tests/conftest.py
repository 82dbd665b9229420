import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built library")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_sessionfinish(session, exitstatus):
    from error_report import write_if_requested

    write_if_requested()


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    return np.load(ROOT / "tests" / "golden" / "ref_helpers.npz")


@pytest.fixture(scope="session")
def lib():
    """The product library, built if needed."""
    from pyroffi_b200 import _lib, build

    if not _lib.LIB_PATH.exists():
        build.build()
    return _lib.load()


@pytest.fixture(scope="session")
def cpu_port():
    """The oracle's C port (built if needed)."""
    import ctypes
    import subprocess

    so = ROOT / "oracle" / "_build" / "libpk_cpu.so"
    if not so.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "cpu"], check=True, capture_output=True)
    return ctypes.CDLL(str(so))

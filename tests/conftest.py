import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def sip_lib():
    """The built C-ABI library (built here if missing)."""
    from sip_b200 import _lib, build

    if not _lib.LIB_PATH.exists():
        build.build()
    return _lib.lib()


@pytest.fixture(scope="session")
def emu():
    """The CPU harness over the kernels' host-device phase functions."""
    from tests.native.build_emu import load

    return load()


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; a gpu-marked test fails loudly without one."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for a gpu-marked test")
    torch.cuda.init()
    return torch

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
    import ctypes

    from tests.native import build_emu

    lib = ctypes.CDLL(str(build_emu.build()))
    c = ctypes
    lib.emu_exec.argtypes = [c.c_int, c.c_int, c.c_int, c.POINTER(c.c_longlong), c.c_longlong, c.c_void_p,
                             c.c_void_p, c.c_char_p, c.c_size_t]
    lib.emu_exec.restype = c.c_int
    lib.emu_fastdiv_check.argtypes = [c.c_void_p, c.c_void_p, c.c_longlong]
    lib.emu_fastdiv_check.restype = c.c_longlong
    lib.emu_radices.argtypes = [c.c_int, c.c_int, c.c_void_p, c.c_int]
    lib.emu_radices.restype = c.c_int
    lib.emu_dft.argtypes = [c.c_int, c.c_int, c.c_void_p]
    lib.emu_dft.restype = c.c_int
    return lib


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; a gpu-marked test fails loudly without one."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for a gpu-marked test")
    torch.cuda.init()
    return torch

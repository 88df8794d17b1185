"""Builds the CPU harness tests/native/libtile_emu.so (test infrastructure).

The harness links the library's planner (sip_b200/csrc/plan.cpp) with
tests/native/tile_emu.cpp, which drives the kernels' host-device phase
functions on the CPU.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
CSRC = ROOT / "sip_b200" / "csrc"
LIB = HERE / "libtile_emu.so"
NVCC = "/usr/local/cuda/bin/nvcc"


def build() -> Path:
    srcs = [HERE / "tile_emu.cpp", CSRC / "plan.cpp", CSRC / "bluestein_host.cpp"]
    deps = srcs + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").rglob("*.h"))
    if LIB.exists() and LIB.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return LIB
    cmd = [NVCC, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared", "-I", str(ROOT / "include"),
           "-I", str(CSRC), *map(str, srcs), "-o", str(LIB)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"harness build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def load():
    """Builds (if stale) and loads the harness with its ctypes signatures."""
    import ctypes as c

    lib = c.CDLL(str(build()))
    lib.emu_exec.argtypes = [c.c_int, c.c_int, c.c_int, c.POINTER(c.c_longlong), c.c_longlong, c.c_void_p,
                             c.c_void_p, c.c_char_p, c.c_size_t]
    lib.emu_exec.restype = c.c_int
    lib.emu_fastdiv_check.argtypes = [c.c_void_p, c.c_void_p, c.c_longlong]
    lib.emu_fastdiv_check.restype = c.c_longlong
    lib.emu_radices.argtypes = [c.c_int, c.c_int, c.c_void_p, c.c_int]
    lib.emu_radices.restype = c.c_int
    lib.emu_dft.argtypes = [c.c_int, c.c_int, c.c_void_p]
    lib.emu_dft.restype = c.c_int
    lib.emu_set_chunk_bytes.argtypes = [c.c_longlong]
    lib.emu_set_chunk_bytes.restype = None
    return lib


if __name__ == "__main__":
    print(build())

"""Build recipe of the B200 FFT library.

Compiles the CUDA kernels for sm_100a and the host C++ into the in-tree
shared library ``sip_b200/libsip_fft.so`` (the C ABI of include/fft_api.h
and include/sip_fft_ext.h).  Objects are cached under ``sip_b200/_build``
and rebuilt when any source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libsip_fft.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-I", str(ROOT / "include"), "-I", str(CSRC)]

# (source, extra defines, object name)
UNITS = [
    ("tile_inst.cu", ["-DSIP_INST_SIGN=-1", "-DSIP_INST_E=16"], "tile_fwd_e16.o"),
    ("tile_inst.cu", ["-DSIP_INST_SIGN=-1", "-DSIP_INST_E=32"], "tile_fwd_e32.o"),
    ("tile_inst.cu", ["-DSIP_INST_SIGN=1", "-DSIP_INST_E=16"], "tile_inv_e16.o"),
    ("tile_inst.cu", ["-DSIP_INST_SIGN=1", "-DSIP_INST_E=32"], "tile_inv_e32.o"),
    *[("sk_shard.cu", [f"-DSIP_SK_SHARD={i}"], f"sk_shard{i}.o") for i in range(8)],
    ("sk_registry.cu", [], "sk_registry.o"),
    ("tile_kernels.cu", [], "tile_kernels.o"),
    ("twiddle.cu", [], "twiddle.o"),
    ("tc_kernel.cu", [], "tc_kernel.o"),
    ("queue.cu", [], "queue.o"),
    ("batch.cpp", [], "batch.o"),
    ("noalloc.cu", [], "noalloc.o"),
    ("shift.cu", [], "shift.o"),
    ("bluestein.cu", [], "bluestein.o"),
    ("bluestein_host.cpp", [], "bluestein_host.o"),
    ("real_kernels.cu", [], "real_kernels.o"),
    ("cluster.cu", [], "cluster.o"),
    ("plan.cpp", [], "plan.o"),
    ("device.cpp", [], "device.o"),
    ("api.cpp", [], "api.o"),
    ("acl_tensor.cpp", [], "acl_tensor.o"),
    ("jit.cpp", [], "jit.o"),
    (str(BUILD / "jit_headers.cpp"), [], "jit_headers.o"),
]

# Kernel headers the run-time compiler (csrc/jit.cpp) builds sk kernels
# from; embedded into the library so that it does not depend on the source
# tree at run time.
JIT_HEADERS = ["sk_kernel.cuh", "sk_modes.h", "fft_core.cuh", "tile_io.cuh"]


def _gen_jit_headers() -> None:
    BUILD.mkdir(exist_ok=True)
    parts = ["// Generated by sip_b200/build.py: kernel headers for csrc/jit.cpp.", "namespace sipfft {",
             f"extern const int kJitHeaderCount = {len(JIT_HEADERS)};",
             "extern const char* const kJitHeaderNames[] = {" + ", ".join(f'"{h}"' for h in JIT_HEADERS) + "};",
             "extern const char* const kJitHeaderTexts[] = {"]
    for h in JIT_HEADERS:
        text = (CSRC / h).read_text()
        if ')sipjit"' in text:
            raise RuntimeError(f"{h} contains the raw-string delimiter")
        parts.append('R"sipjit(' + text + ')sipjit",')
    parts += ["};", "}  // namespace sipfft", ""]
    out = BUILD / "jit_headers.cpp"
    new = "\n".join(parts)
    if not out.exists() or out.read_text() != new:
        out.write_text(new)


def _newest_header() -> float:
    heads = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").rglob("*.h"))
    return max((h.stat().st_mtime for h in heads), default=0.0)


def _deps_mtime(dep: Path, head_mtime: float) -> float:
    """Newest mtime of the headers a unit included at its last compile (the
    compiler's dependency file); every header when there is none."""
    if not dep.exists():
        return head_mtime
    text = dep.read_text().replace("\\\n", " ")
    names = text.split(":", 1)[1].split() if ":" in text else []
    newest = 0.0
    for n in names:
        p = Path(n)
        if not p.exists():
            return head_mtime  # a header went away: rebuild
        newest = max(newest, p.stat().st_mtime)
    return newest


def _compile(src: str, defs: list[str], obj: str, head_mtime: float, verbose: bool) -> str:
    out = BUILD / obj
    dep = BUILD / (obj + ".d")
    s = CSRC / src  # an absolute src (generated under _build) replaces CSRC
    if out.exists() and out.stat().st_mtime >= max(s.stat().st_mtime, _deps_mtime(dep, head_mtime)):
        return f"up to date {obj}"
    cmd = [NVCC, *ARCH, *COMMON, *defs, "-MD", "-MF", str(dep), "-c", str(s), "-o", str(out)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} {defs}:\n{r.stdout}\n{r.stderr}")
    return f"built {obj}" + (("\n" + r.stderr) if verbose else "")


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    _gen_jit_headers()
    head = _newest_header()
    jobs = jobs or max(1, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, d, o, head, verbose) for s, d, o in UNITS]
        for f in futs:
            msg = f.result()
            if verbose:
                print(msg)
    objs = [str(BUILD / o) for _, _, o in UNITS]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *objs, "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)

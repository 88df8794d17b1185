"""ORACLE — CPU checker for the FFT library.  Test infrastructure only:
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import it; the library never does.

Pieces (hicann/sip paths relative to the reference root):

* `golden_*`: the CPU golden "as the reference's tests use it" — numpy.fft
  cast to complex64/float32 with the reference's direction/normalisation
  table (tests/ut/unittest/fft/1d/c2c/c2c_data/gen_data.py:42-47,
  1d/r2c/r2c_data/gen_data.py:42-49, 1d/c2r/c2r_data/gen_data.py:42-49,
  2d/c2c/c2c_2d_data/gen_data_2d.py:64-67): C2C fwd fft, inv
  ifft(norm="forward"); R2C fwd rfft, inv ihfft(norm="forward") =
  conj(rfft); C2R inv irfft(norm="forward"), fwd hfft.
* `fp64_*`: the same transforms in complex128 (the FP64 oracle of
  tests/standalone/fft1d_optimized/run.py:88-105).
* `isclose_mismatches`: numpy-isclose comparison of
  tests/ut/unittest/test_common.h:41-117 (rtol 1e-3, atol 1e-5).
* `lcg_uniform` / `ut_input`: the reference unit tests' fixed-seed inputs
  (tests/ut/framework/test_util/float_util.h:23-36, util.cpp:318-339).
* `kat_input`: the zero / constant / impulse / Nyquist / random patterns
  of tests/standalone/fft1d_optimized/run.py:61-107.
* `stockham_*`: ctypes entry points of the plain-C restatement of the
  reference's Stockham / real pack arithmetic (oracle/stockham.c), and
  `ref_stockham_c2c` of the reference's own Stockham core compiled for
  the CPU (oracle/_ref, present only where the reference sources were).
* `chirp_spectrum` / `pulse`: FP64 pulse compression IFFT(FFT(x) * F), the
  matched-filter chain the reference composes from asdFftExecC2C and asdMul
  (include/base_api.h:29), with the linear-chirp pulse of the serving
  workload.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
REF_PATH = HERE / "_ref" / "libref_stockham.so"

C2C, C2R, R2C = 0x10, 0x11, 0x12
FORWARD, INVERSE = 0x10, 0x11

_lib = None
_ref = None


def build() -> None:
    """Compiles the C restatement (and oracle/_ref when the reference is here)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        l = ctypes.CDLL(str(LIB_PATH))
        i64, vp = ctypes.c_int64, ctypes.c_void_p
        for suf in ("f32", "f64"):
            for op in ("c2c", "r2c", "c2r"):
                fn = getattr(l, f"orc_{op}_{suf}")
                fn.argtypes = [i64, ctypes.c_int, i64, vp, vp]
                fn.restype = ctypes.c_int
        l.orc_lcg_uniform.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_float, ctypes.c_float, i64, vp]
        l.orc_set_threads.argtypes = [ctypes.c_int]
        l.orc_get_threads.restype = ctypes.c_int
        _lib = l
    return _lib


def ref_lib():
    """The reference's own Stockham core (None when it was not built here)."""
    global _ref
    if _ref is None and REF_PATH.exists():
        l = ctypes.CDLL(str(REF_PATH))
        l.ref_stockham_c2c.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        l.ref_stockham_c2c.restype = ctypes.c_int
        _ref = l
    return _ref


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ----------------------------------------------------------------- inputs
def lcg_uniform(count: int, lo: float = -300.0, hi: float = 300.0, state: int = 2026) -> np.ndarray:
    out = np.empty(count, dtype=np.float32)
    st = ctypes.c_uint32(state)
    lib().orc_lcg_uniform(ctypes.byref(st), lo, hi, count, out.ctypes.data)
    return out


def ut_input(shape, dtype) -> np.ndarray:
    """Input tensor of the reference unit tests: LCG from state 2026, U[-300, 300);
    complex tensors interleave real/imag draws (util.cpp:324-339)."""
    n = int(np.prod(shape))
    if np.dtype(dtype) == np.complex64:
        return lcg_uniform(2 * n).view(np.complex64).reshape(shape)
    return lcg_uniform(n).reshape(shape)


def kat_input(pattern: str, op: int, n: int, batch: int, dim: int = 1, direction: int = FORWARD):
    """Known-answer inputs of run.py:61-107 (seed 20261029 + n) and their FP64 golden."""
    shape = (batch,) + (n,) * dim
    axes = tuple(range(-dim, 0))
    rng = np.random.default_rng(20261029 + n)
    raw = rng.standard_normal(shape, dtype=np.float32)
    if pattern == "zero":
        raw.fill(0)
    elif pattern == "constant":
        raw.fill(1)
    elif pattern == "impulse":
        raw.fill(0)
        raw.reshape(-1, n)[:, 1] = 1
    elif pattern == "nyquist":
        raw[...] = np.where(np.arange(n) % 2, -1, 1)
    if op == C2C:
        imag = rng.standard_normal(shape, dtype=np.float32) if pattern == "random" else raw
        x = (raw + 1j * imag).astype(np.complex64)
    elif op == R2C:
        x = raw
    else:
        x = np.fft.rfftn(raw.astype(np.float64), axes=axes).astype(np.complex64)
    return x, fp64(op, direction, x, (n,) * dim)


# ---------------------------------------------------------------- goldens
def fp64(op: int, direction: int, x: np.ndarray, sizes) -> np.ndarray:
    """FP64 oracle over the trailing len(sizes) axes."""
    sizes = tuple(int(s) for s in sizes)
    axes = tuple(range(-len(sizes), 0))
    if op == C2C:
        z = x.astype(np.complex128)
        return np.fft.fftn(z, axes=axes) if direction == FORWARD else np.fft.ifftn(z, axes=axes, norm="forward")
    if op == R2C:
        g = np.fft.rfftn(x.astype(np.float64), axes=axes)
        return g if direction == FORWARD else np.conj(g)
    z = x.astype(np.complex128)
    if direction == FORWARD:
        z = np.conj(z)
    return np.fft.irfftn(z, s=sizes, axes=axes, norm="forward")


def chirp_spectrum(n: int) -> np.ndarray:
    """Spectrum of a linear chirp c[t] = exp(i pi t^2 / L), L = max(1, n // 4),
    zero-padded to n (the pulse-compression workload's transmitted pulse)."""
    L = max(1, n // 4)
    c = np.zeros(n, np.complex128)
    t = np.arange(L)
    c[:L] = np.exp(1j * np.pi * t * t / L)
    return np.fft.fft(c)


def pulse(x: np.ndarray, filt: np.ndarray, conj: bool = False, scale: bool = False) -> np.ndarray:
    """FP64 pulse compression of each row: IFFT(FFT(x) * F), unnormalised
    (times 1/n with `scale`), F conjugated with `conj` (matched filter)."""
    n = x.shape[-1]
    f = np.conj(filt.astype(np.complex128)) if conj else filt.astype(np.complex128)
    y = np.fft.ifft(np.fft.fft(x.astype(np.complex128), axis=-1) * f, axis=-1)
    return y if scale else y * n


def shift2d(x: np.ndarray, row: int, col: int, batch: int, dist: int, inverse: bool, scale: float = 1.0):
    """Golden of asdFftShift / asdIfftShift (tests/ut/unittest/fft/fftshift/
    fftshift_data/gen_data.py): each slice s (elements s*dist ..) rolled by
    ((row+1)//2, (col+1)//2), or by (row//2, col//2) and scaled for the
    inverse; output slices contiguous."""
    if dist <= 0:
        dist = row * col
    out = np.empty((batch, row, col), np.complex64)
    sr, sc = (row // 2, col // 2) if inverse else ((row + 1) // 2, (col + 1) // 2)
    for b in range(batch):
        sl = x[b * dist:b * dist + row * col].reshape(row, col)
        r = np.roll(sl, (sr, sc), axis=(0, 1))
        out[b] = (r * np.float32(scale)).astype(np.complex64) if inverse and scale != 1.0 else r
    return out


def golden(op: int, direction: int, x: np.ndarray, sizes) -> np.ndarray:
    """numpy.fft at the input's precision, cast like the reference's gen_data.py."""
    sizes = tuple(int(s) for s in sizes)
    if len(sizes) == 1:
        n = sizes[0]
        if op == C2C:
            g = np.fft.fft(x, n=n, axis=-1) if direction == FORWARD else np.fft.ifft(x, n=n, axis=-1, norm="forward")
            return g.astype(np.complex64)
        if op == R2C:
            g = np.fft.rfft(x, n=n, axis=-1) if direction == FORWARD else np.fft.ihfft(x, n=n, axis=-1, norm="forward")
            return g.astype(np.complex64)
        g = np.fft.hfft(x, n=n, axis=-1) if direction == FORWARD else np.fft.irfft(x, n=n, axis=-1, norm="forward")
        return g.astype(np.float32)
    axes = tuple(range(-len(sizes), 0))
    if op == C2C:
        g = np.fft.fftn(x, axes=axes) if direction == FORWARD else np.fft.ifftn(x, axes=axes, norm="forward")
        return g.astype(np.complex64)
    return fp64(op, direction, x, sizes).astype(np.complex64 if op == R2C else np.float32)


def isclose_mismatches(out: np.ndarray, gold: np.ndarray, rtol: float = 1e-3, atol: float = 1e-5) -> int:
    """Elements failing |out - gold| <= atol + rtol |gold| (NaN fails)."""
    o = out.astype(np.complex128).ravel()
    g = gold.astype(np.complex128).ravel()
    diff = np.abs(o - g)
    return int(np.count_nonzero(~(diff <= atol + rtol * np.abs(g))))


def ref_check_mismatches(out: np.ndarray, gold: np.ndarray) -> int:
    """The reference's elementwise check (rtol 1e-3, atol 1e-5) with the
    absolute tolerance floored at 1e-6 of the largest golden magnitude.

    An FP32 FFT carries errors near 1e-7 of the spectrum's peak on every
    bin, so bins a thousand times below the peak cannot meet a 1e-3
    relative bound: the C restatement of the reference's FP32 Stockham
    arithmetic (stockham.c) misses it on 2 of the 32768 outputs of the
    reference's C2R N=32768 forward case, at rel-L2 1.5e-7.  The floor is
    the 1e-6 relative-error bar of this library."""
    peak = float(np.abs(gold.astype(np.complex128)).max()) if gold.size else 0.0
    return isclose_mismatches(out, gold, 1e-3, max(1e-5, 1e-6 * peak))


def rel_l2(out: np.ndarray, ref: np.ndarray) -> float:
    d = np.linalg.norm((out.astype(np.complex128) - ref.astype(np.complex128)).ravel())
    n = np.linalg.norm(ref.astype(np.complex128).ravel())
    return float(d / n) if n else float(d)


def max_bin_err(out: np.ndarray, ref: np.ndarray) -> float:
    """max |out - ref| / max |ref| (spectral max-bin error)."""
    r = np.abs(ref.astype(np.complex128)).max()
    e = np.abs(out.astype(np.complex128) - ref.astype(np.complex128)).max()
    return float(e / r) if r else float(e)


# ------------------------------------------------ C restatement (ctypes)
def stockham(op: int, direction: int, x: np.ndarray, n: int, fp64_math: bool = False) -> np.ndarray:
    """1D transform of the rows of x with the C restatement (float or double arithmetic)."""
    inv = 1 if direction == INVERSE else 0
    ft, ct = (np.float64, np.complex128) if fp64_math else (np.float32, np.complex64)
    suf = "f64" if fp64_math else "f32"
    l = lib()
    if op == C2C:
        src = np.ascontiguousarray(x, dtype=ct)
        batch = src.size // n
        out = np.empty_like(src)
        getattr(l, f"orc_c2c_{suf}")(n, inv, batch, src.ctypes.data, out.ctypes.data)
        return out
    if op == R2C:
        src = np.ascontiguousarray(x, dtype=ft)
        batch = src.size // n
        out = np.empty(src.shape[:-1] + (n // 2 + 1,), dtype=ct)
        getattr(l, f"orc_r2c_{suf}")(n, inv, batch, src.ctypes.data, out.ctypes.data)
        return out
    src = np.ascontiguousarray(x, dtype=ct)
    batch = src.size // (n // 2 + 1)
    out = np.empty(src.shape[:-1] + (n,), dtype=ft)
    getattr(l, f"orc_c2r_{suf}")(n, inv, batch, src.ctypes.data, out.ctypes.data)
    return out


def ref_stockham_c2c(x: np.ndarray, inverse: bool = False):
    """The reference's own Stockham core on complex64 rows (None if unavailable
    or the length is outside its admission)."""
    l = ref_lib()
    if l is None:
        return None
    src = np.ascontiguousarray(x, dtype=np.complex64)
    m = src.shape[-1]
    out = np.empty_like(src)
    rc = l.ref_stockham_c2c(m, 1 if inverse else 0, src.size // m, src.ctypes.data, out.ctypes.data)
    return None if rc != 0 else out


def cpu_info() -> dict:
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cores": os.cpu_count(), "model": model}

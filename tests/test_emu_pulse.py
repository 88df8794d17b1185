"""Fused pulse compression (IFFT(FFT(x) * F)) through the CPU harness.

The harness runs the planner's steps with the kernels' own phase functions
thread by thread: one fused tile step up to n = 16384, the three-pass
four-step form above it.  Results are checked against the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

REL_L2_TOL = 1e-6

CASES = [(256, 5), (1000, 3), (4096, 2), (6000, 2), (16384, 1), (20000, 2), (65536, 1), (1 << 18, 1)]


def run_pulse(emu, n, batch, x, filt, flags):
    emu.emu_exec_pulse.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    emu.emu_exec_pulse.restype = ctypes.c_int
    out = np.zeros_like(x)
    f = np.ascontiguousarray(filt.astype(np.complex64))
    desc = ctypes.create_string_buffer(1 << 16)
    rc = emu.emu_exec_pulse(n, batch, f.ctypes.data, flags, x.ctypes.data, out.ctypes.data, desc, len(desc))
    return rc, out, desc.value.decode()


def signal(n, batch, seed):
    """Delayed chirps plus complex noise (sigma 0.1 per component)."""
    rng = np.random.default_rng(seed)
    L = max(1, n // 4)
    t = np.arange(L)
    c = np.exp(1j * np.pi * t * t / L)
    x = 0.1 * (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n)))
    for b in range(batch):
        d = int(rng.integers(0, n - L + 1))
        x[b, d:d + L] += c
    return x.astype(np.complex64)


@pytest.mark.parametrize("n,batch", CASES)
@pytest.mark.parametrize("flags", [0, 1, 3])
def test_pulse_matches_fp64(emu, n, batch, flags):
    x = signal(n, batch, 20261203 + n)
    filt = O.chirp_spectrum(n)
    rc, out, desc = run_pulse(emu, n, batch, x, filt, flags)
    assert rc == 0, desc
    want = O.pulse(x, filt, conj=bool(flags & 1), scale=bool(flags & 2))
    assert O.rel_l2(out, want) <= REL_L2_TOL, desc
    kinds = [s["what"].split(" n=")[0] for s in __import__("json").loads(desc)["steps"]]
    assert kinds == (["pulse rows"] if n <= 16384 else ["four-step A", "pulse rows", "pulse inverse columns"])
    # the harness's size-specialized pulse tiles (rows of 1000; pass P of
    # 2^18 = 512 x 512 with cross twiddles) run where they apply
    pulse = [s for s in __import__("json").loads(desc)["steps"] if s["what"].startswith("pulse rows")]
    if n in (1000, 1 << 18):
        assert pulse[0]["sk"], desc


def test_matched_filter_peaks_at_delay(emu):
    """The matched-filter output of a delayed chirp peaks at the delay."""
    n, L, d = 4096, 1024, 777
    t = np.arange(L)
    x = np.zeros((1, n), np.complex64)
    x[0, d:d + L] = np.exp(1j * np.pi * t * t / L)
    rc, out, _ = run_pulse(emu, n, 1, x, O.chirp_spectrum(n), 3)
    assert rc == 0
    assert int(np.argmax(np.abs(out[0]))) == d

"""Run-time specialized tile kernels (csrc/jit.cpp).

Lengths without a compiled size-specialized kernel get one compiled by
NVRTC from the library's own kernel headers.  CPU tests: the planner's
choice (describe) and that the generated source compiles for every tile
mode and real-transform operation (NVRTC needs no GPU).  GPU tests: parity
of the compiled kernels with the FP64 oracle, forced on at small batches
with SIP_FFT_HINT_RUNTIME_COMPILE = 1, against the generic kernel too.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle, shapes

REL_L2_TOL = 1e-6

OP_C2C, OP_R2C_HALF, OP_C2R_HALF, OP_R2C_PAIR, OP_C2R_PAIR, OP_PC = 0, 1, 2, 3, 4, 7
ROWS, COLS, ROWS_T = 0, 1, 2


@pytest.fixture()
def jit_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("SIP_FFT_JIT_CACHE", str(tmp_path / "jit"))
    return tmp_path / "jit"


def _plan(op, direction, sizes, batch, jit):
    from sip_b200.fft import FftHandle, check

    h = FftHandle()
    check(h.set_hint(L.SIP_FFT_HINT_RUNTIME_COMPILE, jit), "hint")
    rc = {1: lambda: h.make_plan_1d(sizes[0], op, direction, batch),
          2: lambda: h.make_plan_2d(sizes[0], sizes[1], op, direction, batch)}[len(sizes)]()
    check(rc, "make plan")
    return h


def _nvrtc_present():
    return L.lib().sipFftJitCompileCheck(OP_C2C, ROWS, -1, 0, 3840, 64) != L.ACL_ERROR_API_NOT_SUPPORT


@pytest.mark.parametrize("op,direction,n,batch,jit,expect", [
    (O.C2C, O.FORWARD, 3840, 8192, 0, True),    # 31M values: compiled at run time by default
    (O.C2C, O.FORWARD, 3840, 16, 0, False),     # small step: generic kernel
    (O.C2C, O.FORWARD, 3840, 16, 1, True),      # forced on
    (O.C2C, O.FORWARD, 3840, 8192, 2, False),   # forced off
    (O.C2C, O.FORWARD, 4096, 8192, 1, False),   # a compiled kernel exists: no run-time one
    (O.R2C, O.FORWARD, 6688, 8, 1, True),
    (O.C2R, O.INVERSE, 2001, 8, 1, True),       # odd real length: row pairs
])
def test_planner_choice(op, direction, n, batch, jit, expect):
    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    h = _plan(op, direction, [n], batch, jit)
    steps = [s for s in h.describe()["steps"] if "jit" in s]
    h.destroy()
    if jit == 0 and expect:
        # the default compiles a new configuration in the background: this
        # plan may run the generic kernel, one made after the wait does not
        assert L.lib().sipFftJitWait(300000) == L.ACL_SUCCESS
        h = _plan(op, direction, [n], batch, jit)
        steps = [s for s in h.describe()["steps"] if "jit" in s]
        h.destroy()
    assert any(s["jit"] for s in steps) == expect, steps
    for s in steps:
        if s["jit"]:
            assert s["sk"] and 32 <= s["threads"] <= 512 and s["threads"] % 32 == 0
            assert int(np.prod(s["radices"])) == s["n"] and max(s["radices"]) <= 32


def test_hint_validation():
    from sip_b200.fft import FftHandle

    assert L.lib().sipFftJitWait(-1) == L.ACL_ERROR_INVALID_PARAM
    h = FftHandle()
    assert h.set_hint(L.SIP_FFT_HINT_RUNTIME_COMPILE, 3) == L.ACL_ERROR_INVALID_PARAM
    assert h.set_hint(L.SIP_FFT_HINT_RUNTIME_COMPILE, 2) == L.ACL_SUCCESS
    h.destroy()


# One configuration per operation and tile mode (compiled on the CPU).
COMPILE_CASES = [
    (OP_C2C, ROWS, -1, 0, 3840, 8192),
    (OP_C2C, ROWS, 1, 0, 2944, 8192),       # radix 23
    (OP_C2C, ROWS, -1, 0, 16337, 3),        # 17 x 31 x 31: no room for the staged twiddles beside the tile
    (OP_C2C, COLS, -1, 1, 243, 9000),       # four-step column pass with cross twiddles
    (OP_C2C, ROWS_T, 1, 0, 625, 9000),      # four-step row pass, transposed store
    (OP_R2C_HALF, ROWS, -1, 0, 3344, 8192),
    (OP_C2R_HALF, ROWS, 1, 0, 3344, 8192),
    (OP_R2C_PAIR, ROWS, -1, 0, 2001, 1000),
    (OP_C2R_PAIR, ROWS, 1, 0, 2001, 1000),
    (OP_PC, ROWS, 1, 0, 10800, 8192),       # pulse compression tile (Bluestein's convolution)
    (OP_PC, ROWS, 1, 1, 225, 9000),         # four-step pulse pass P
]


@pytest.mark.parametrize("op,mode,sign,tw4,n,transforms", COMPILE_CASES)
def test_generated_source_compiles(jit_cache, op, mode, sign, tw4, n, transforms):
    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    assert L.lib().sipFftJitCompileCheck(op, mode, sign, tw4, n, transforms) == L.ACL_SUCCESS


def test_disk_cache(tmp_path):
    """A fresh process compiles into the cache directory; a second process
    finds every cubin there and compiles nothing new."""
    import subprocess
    import sys

    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    cache = tmp_path / "jit"
    code = ("import sys; sys.path.insert(0, %r); from sip_b200 import _lib as L; "
            "sys.exit(L.lib().sipFftJitCompileCheck(0, 0, -1, 0, 3840, 8192))" % os.getcwd())
    env = dict(os.environ, SIP_FFT_JIT_CACHE=str(cache))
    assert subprocess.run([sys.executable, "-c", code], env=env).returncode == 0
    first = {p.name: p.stat().st_mtime_ns for p in cache.glob("sk_*.cubin")}
    assert first, "cubin not cached"
    assert subprocess.run([sys.executable, "-c", code], env=env).returncode == 0
    assert {p.name: p.stat().st_mtime_ns for p in cache.glob("sk_*.cubin")} == first


def test_unsupported_configurations():
    lib = L.lib()
    assert lib.sipFftJitCompileCheck(OP_C2C, ROWS, -1, 0, 2656, 64) == L.ACL_ERROR_API_NOT_SUPPORT  # factor 83
    assert lib.sipFftJitCompileCheck(OP_R2C_HALF, COLS, -1, 0, 1000, 64) == L.ACL_ERROR_API_NOT_SUPPORT
    assert lib.sipFftJitCompileCheck(OP_C2C, ROWS, -1, 0, 32768, 64) == L.ACL_ERROR_API_NOT_SUPPORT  # > one tile


def _input(op, n_sizes, batch, seed):
    rng = np.random.default_rng(seed)
    ishape, idt, _, _ = shapes(op, n_sizes, batch)
    if op == O.C2R:
        return np.fft.rfftn(rng.uniform(-1, 1, (batch, *n_sizes)), axes=tuple(range(1, len(n_sizes) + 1))
                            ).astype(np.complex64).reshape(ishape)
    if idt == np.float32:
        return rng.uniform(-1, 1, ishape).astype(np.float32)
    return (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64)


def _gpu(torch, op, direction, sizes, batch, x, jit):
    from sip_b200.fft import check

    _, _, oshape, odt = shapes(op, sizes, batch)
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yt = torch.zeros(oshape, dtype=torch.complex64 if odt == np.complex64 else torch.float32, device="cuda")
    h = _plan(op, direction, sizes, batch, jit)
    used = any(s.get("jit") for s in h.describe()["steps"])
    h.bind_workspace()
    s = torch.cuda.Stream()
    check(h.set_stream(s), "stream")
    fn = {O.C2C: h.exec_c2c, O.R2C: h.exec_r2c, O.C2R: h.exec_c2r}[op]
    settle()
    check(fn(xt, yt), "exec")
    check(h.synchronize(), "sync")
    out = yt.cpu().numpy()
    h.destroy()
    return out, used


# (op, direction, sizes, batch): rows of lengths without compiled kernels,
# odd real lengths (pairs), 2-D column passes and four-step lengths.
GPU_CASES = [
    (O.C2C, O.FORWARD, [3840], 37), (O.C2C, O.INVERSE, [2016], 21), (O.C2C, O.FORWARD, [544], 50),
    (O.C2C, O.INVERSE, [6720], 9), (O.C2C, O.FORWARD, [8160], 5), (O.C2C, O.INVERSE, [2944], 11),
    (O.C2C, O.FORWARD, [16337], 3), (O.C2C, O.INVERSE, [5400], 7), (O.C2C, O.FORWARD, [96], 300),
    (O.R2C, O.FORWARD, [6688], 13), (O.C2R, O.INVERSE, [6720], 13), (O.R2C, O.INVERSE, [5000], 9),
    (O.R2C, O.FORWARD, [2001], 15), (O.C2R, O.INVERSE, [2001], 15), (O.C2R, O.FORWARD, [729], 40),
    (O.C2C, O.FORWARD, [243, 300], 3), (O.C2C, O.INVERSE, [625, 96], 2),
    (O.C2C, O.FORWARD, [3840 * 64], 2), (O.C2C, O.INVERSE, [243 * 625], 2),
    (O.R2C, O.FORWARD, [2 * 3840 * 48], 2), (O.C2R, O.INVERSE, [2 * 3840 * 48], 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("op,direction,sizes,batch", GPU_CASES)
def test_jit_parity(cuda, jit_cache, op, direction, sizes, batch):
    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    x = _input(op, sizes, batch, seed=sum(sizes) + batch)
    out, used = _gpu(cuda, op, direction, sizes, batch, x, jit=1)
    assert used, "no step was compiled at run time"
    err = O.rel_l2(out, O.fp64(op, direction, x, sizes))
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}"
    gen, used_gen = _gpu(cuda, op, direction, sizes, batch, x, jit=2)
    assert not used_gen
    assert O.rel_l2(out, gen) <= 2 * REL_L2_TOL


# Pulse compression (OP_PC tiles: forward FFT, filter, inverse FFT in shared
# memory) compiled at run time: one-tile rows and the four-step pass P.
@pytest.mark.gpu
@pytest.mark.parametrize("n,batch", [(1000, 33), (10800, 3), (3840 * 64, 2)])
@pytest.mark.parametrize("flags", [1, 3])
def test_jit_pulse(cuda, jit_cache, n, batch, flags):
    from sip_b200.fft import FftHandle, check
    from tests.test_emu_pulse import signal

    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    torch = cuda
    x = signal(n, batch, 20261203 + n)
    filt = O.chirp_spectrum(n)
    xt = torch.from_numpy(x).cuda()
    ft = torch.from_numpy(filt.astype(np.complex64)).cuda()
    yt = torch.zeros_like(xt)
    h = FftHandle()
    check(h.set_hint(L.SIP_FFT_HINT_RUNTIME_COMPILE, 1), "hint")
    check(h.make_plan_pulse_1d(n, batch, ft.data_ptr(), flags), "sipFftMakePlanPulse1D")
    assert any(s.get("jit") and s.get("op") == 7 for s in h.describe()["steps"])
    h.bind_workspace()
    s = torch.cuda.Stream()
    check(h.set_stream(s), "stream")
    settle()
    check(h.exec_c2c(xt, yt), "exec")
    s.synchronize()
    want = O.pulse(x, filt, conj=bool(flags & 1), scale=bool(flags & 2))
    assert O.rel_l2(yt.cpu().numpy(), want) <= REL_L2_TOL
    h.destroy()


# Bluestein lengths: the convolution runs as a run-time compiled OP_PC tile.
@pytest.mark.gpu
@pytest.mark.parametrize("op,direction,n,batch", [(O.R2C, O.FORWARD, 5312, 6), (O.C2R, O.INVERSE, 5344, 6),
                                                  (O.C2C, O.INVERSE, 6752, 5), (O.C2C, O.FORWARD, 20011, 2)])
def test_jit_bluestein(cuda, jit_cache, op, direction, n, batch):
    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    x = _input(op, [n], batch, seed=n)
    out, used = _gpu(cuda, op, direction, [n], batch, x, jit=1)
    assert used
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}"


def _random_lengths(seed, count):
    """Lengths up to one tile whose factors are all <= 31 and that have no
    compiled kernel, drawn with a fixed seed."""
    rng = np.random.default_rng(seed)
    primes = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31]
    compiled = {50, 256, 500, 1000, 1024, 2048, 2187, 3000, 4096, 6000, 8192}
    out = []
    while len(out) < count:
        n = 1
        for _ in range(int(rng.integers(2, 6))):
            n *= int(rng.choice(primes, p=[.3, .2, .15, .1, .05, .05, .05, .04, .02, .02, .02]))
        if 64 <= n <= 16384 and n not in compiled and n not in out:
            out.append(n)
    return out


# Randomly drawn lengths with the run-time kernels forced on: C2C rows both
# directions, R2C / C2R (half length for even n, row pairs for odd n).
@pytest.mark.gpu
@pytest.mark.parametrize("n", _random_lengths(20261203, 12))
@pytest.mark.parametrize("op,direction", [(O.C2C, O.FORWARD), (O.C2C, O.INVERSE), (O.R2C, O.FORWARD),
                                          (O.C2R, O.INVERSE)])
def test_jit_random_lengths(cuda, jit_cache, n, op, direction):
    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    batch = 7
    x = _input(op, [n], batch, seed=n + op)
    out, used = _gpu(cuda, op, direction, [n], batch, x, jit=1)
    assert used
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"n={n} rel_l2 vs FP64 {err:.3e}"


def test_background_compile_exit_and_fork(tmp_path):
    """A process may exit while a background compilation runs, and a child
    forked while the compiler's worker threads exist (their state may have
    been copied mid-compilation) compiles nothing: its plans run the generic
    kernel, and the parent goes on compiling."""
    import subprocess
    import sys

    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    code = r'''
import os, sys
sys.path.insert(0, %r)
from sip_b200 import _lib as L
from sip_b200.fft import FftHandle
def plan(n):
    h = FftHandle()
    assert h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 4096) == 0
    jit = any(s.get("jit") for s in h.describe()["steps"])
    h.destroy()
    return jit
plan(3780)                      # starts the workers and a background compilation
pid = os.fork()
if pid == 0:
    ok = not plan(3960) and L.lib().sipFftJitWait(1000) == 0 and not plan(3960)
    os._exit(0 if ok else 3)
_, status = os.waitpid(pid, 0)
assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0, status
plan(4200)
assert L.lib().sipFftJitWait(300000) == 0 and plan(4200)
plan(4320)                      # leave one running at exit
''' % os.getcwd()
    env = dict(os.environ, SIP_FFT_JIT_CACHE=str(tmp_path / "jit"))
    r = subprocess.run([sys.executable, "-W", "ignore", "-c", code], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


def test_exit_while_compiling_many_times(tmp_path):
    """Processes that exit a fraction of a second after starting background
    compilations (four steps, cold cache) exit cleanly every time.  Before the
    compiler was warmed up ahead of the exit-time drain, some of these exits
    crashed: the compiler's own teardown ran while a worker still compiled."""
    import subprocess
    import sys

    if not _nvrtc_present():
        pytest.skip("NVRTC not available")
    code = r'''
import sys, time
sys.path.insert(0, %r)
from sip_b200 import _lib as L
from sip_b200.fft import FftHandle
for n, b in ((1 << 21, 64), (184320, 16)):   # four-step lengths without compiled kernels
    h = FftHandle()
    assert h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, b) == 0
time.sleep(float(sys.argv[1]))
''' % os.getcwd()
    for i, delay in enumerate((0.0, 0.05, 0.1, 0.2, 0.3, 0.4, 0.5, 0.7)):
        env = dict(os.environ, SIP_FFT_JIT_CACHE=str(tmp_path / f"jit{i}"))
        r = subprocess.run([sys.executable, "-W", "ignore", "-c", code, str(delay)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, (delay, r.returncode, r.stderr[-2000:])

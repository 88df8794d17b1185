"""Tensor-core split-precision form on a B200 (tcgen05, BF16 x3 split,
FP32 accumulation): results match the FP64 oracle at the FP32 path's
accuracy for both input families of the precision benchmark, and no
bounded device wait ran out."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle, random_input

pytestmark = pytest.mark.gpu
REL_L2_TOL = 1e-6


def _run(torch, n, batch, direction, x, mode):
    from sip_b200.fft import FftHandle, check

    dev = torch.device("cuda")
    xt = torch.from_numpy(x).to(dev)
    yt = torch.empty_like(xt)
    with FftHandle() as h:
        check(h.set_compute_mode(mode), "set mode")
        check(h.make_plan_1d(n, O.C2C, direction, batch), "plan")
        h.bind_workspace(dev)
        s = torch.cuda.Stream()
        check(h.set_stream(s), "stream")
        settle()
        check(h.exec_c2c(xt, yt), "exec")
        check(h.synchronize(), "sync")
        desc = h.describe()
    err = ctypes.c_uint(0)
    check(L.lib().sipFftTakeDeviceErrors(ctypes.byref(err)), "device errors")
    assert err.value == 0, "a tensor-core wait ran out"
    return yt.cpu().numpy(), desc


def sinusoids(n, batch, seed):
    """Family B: 8 complex sinusoids, amplitudes spanning 60 dB, + N(0, 1e-6) noise."""
    rng = np.random.default_rng(seed)
    t = np.arange(n)
    x = np.zeros((batch, n), np.complex128)
    for i in range(8):
        f = rng.uniform(0, n, (batch, 1))
        ph = rng.uniform(0, 2 * np.pi, (batch, 1))
        x += 10 ** (-3 * i / 7) * np.exp(1j * (2 * np.pi * ((f * t) % n) / n + ph))
    x += rng.normal(0, 1e-6, (batch, n)) + 1j * rng.normal(0, 1e-6, (batch, n))
    return x.astype(np.complex64)


@pytest.mark.parametrize("n,batch", [(256, 37), (65536, 6)])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
@pytest.mark.parametrize("family", ["noise", "sinusoids"])
def test_tensor_core_split_accuracy(cuda, n, batch, direction, family):
    x = random_input(O.C2C, [n], batch, seed=n) if family == "noise" else sinusoids(n, batch, 20261029 + n)
    out, desc = _run(cuda, n, batch, direction, x, L.SIP_FFT_COMPUTE_TC_SPLIT)
    assert all("tensor-core" in s["what"] for s in desc["steps"]), desc
    ref = O.fp64(O.C2C, direction, x, [n])
    err = O.rel_l2(out, ref)
    fp32, _ = _run(cuda, n, batch, direction, x, L.SIP_FFT_COMPUTE_FP32)
    err32 = O.rel_l2(fp32, ref)
    assert err <= REL_L2_TOL, err
    # the split form keeps FP32-level accuracy (within 2x of the FP32 path)
    assert err <= 2 * err32 + 1e-8, (err, err32)
    assert O.max_bin_err(out, ref) <= 1e-6

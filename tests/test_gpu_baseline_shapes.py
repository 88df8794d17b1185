"""Parity at the benchmark's own shapes, on a B200, through the C ABI.

The configurations the measurement quotes run here at their full sizes:
1-D C2C 4096 x 256; 2-D C2C 2048 x 2048 x 8 and 3-D C2C 256^3, forward and
inverse; 1-D C2C 65536 x 4096 in the FP32 and the tensor-core split form on
both input families of the precision measurement (i.i.d. N(0, 1), and eight
complex sinusoids spanning 60 dB plus N(0, 1e-6) noise).  Inputs are made on
the device from a seed; the FP64 oracle checks every transform of the small
configurations and a sample of whole transforms of the large ones (rel-L2 <=
1e-6, the library's bar, and the max-bin error for the precision form).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-6
SEED = 20261029


def _plan(sizes, direction, batch, stream, mode=None):
    from sip_b200.fft import FftHandle, check

    h = FftHandle()
    if mode is not None:
        check(h.set_compute_mode(mode), "sipFftSetComputeMode")
    if len(sizes) == 1:
        check(h.make_plan_1d(sizes[0], L.ASCEND_FFT_C2C, direction, batch), "asdFftMakePlan1D")
    elif len(sizes) == 2:
        check(h.make_plan_2d(sizes[0], sizes[1], L.ASCEND_FFT_C2C, direction, batch), "asdFftMakePlan2D")
    else:
        check(h.make_plan_3d(*sizes, L.ASCEND_FFT_C2C, direction, batch), "asdFftMakePlan3D")
    h.bind_workspace()
    check(h.set_stream(stream), "asdFftSetStream")
    return h


def _noise(torch, shape, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.complex(torch.randn(shape, generator=g, device="cuda"),
                         torch.randn(shape, generator=g, device="cuda"))


def _run(torch, h, x, stream):
    from sip_b200.fft import check

    y = torch.empty_like(x)
    torch.cuda.synchronize()
    check(h.exec_c2c(x, y), "asdFftExecC2C")
    stream.synchronize()
    return y


@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
@pytest.mark.parametrize("sizes,batch,sample", [([4096], 256, None), ([2048, 2048], 8, [0, 5, 7]),
                                                ([256, 256, 256], 1, [0])])
def test_c2c_benchmark_shapes(cuda, direction, sizes, batch, sample):
    torch = cuda
    s = torch.cuda.Stream()
    x = _noise(torch, (batch, *sizes), SEED + sizes[0])
    h = _plan(sizes, direction, batch, s)
    y = _run(torch, h, x, s)
    h.destroy()
    rows = list(range(batch)) if sample is None else sample
    idx = torch.tensor(rows, device="cuda")
    xs = x.index_select(0, idx).cpu().numpy()
    ys = y.index_select(0, idx).cpu().numpy()
    err = O.rel_l2(ys, O.fp64(O.C2C, direction, xs, sizes))
    assert err <= REL_L2_TOL, f"{sizes} x {batch}: rel_l2 {err:.3e}"


def _sinusoids(torch, batch, n, seed):
    """Eight complex sinusoids per row at random frequencies, amplitudes
    10^(-3 i / 7) (60 dB span), random phases, plus N(0, 1e-6) noise."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    t = torch.arange(n, device="cuda", dtype=torch.float64)
    acc = torch.zeros((batch, n), dtype=torch.complex128, device="cuda")
    for i in range(8):
        f = torch.rand((batch, 1), generator=g, device="cuda", dtype=torch.float64) * n
        ph = torch.rand((batch, 1), generator=g, device="cuda", dtype=torch.float64) * 2 * math.pi
        acc += (10 ** (-3 * i / 7)) * torch.exp(1j * (2 * math.pi * torch.remainder(f * t, n) / n + ph))
    acc += 1e-6 * torch.complex(torch.randn((batch, n), generator=g, device="cuda", dtype=torch.float64),
                                torch.randn((batch, n), generator=g, device="cuda", dtype=torch.float64))
    return acc.to(torch.complex64)


@pytest.mark.parametrize("family", ["noise", "sinusoids"])
@pytest.mark.parametrize("mode", [L.SIP_FFT_COMPUTE_FP32, L.SIP_FFT_COMPUTE_TC_SPLIT])
def test_precision_form_full_batch(cuda, family, mode):
    torch = cuda
    n, batch = 65536, 4096
    s = torch.cuda.Stream()
    x = _noise(torch, (batch, n), SEED + n) if family == "noise" else _sinusoids(torch, batch, n, SEED + n)
    h = _plan([n], O.FORWARD, batch, s, mode)
    y = _run(torch, h, x, s)
    h.destroy()
    idx = torch.tensor([0, 1, 777, 2048, 4095], device="cuda")
    xs = x.index_select(0, idx).cpu().numpy()
    ys = y.index_select(0, idx).cpu().numpy()
    ref = O.fp64(O.C2C, O.FORWARD, xs, [n])
    err = O.rel_l2(ys, ref)
    assert err <= REL_L2_TOL, f"{family} mode {mode}: rel_l2 {err:.3e}"
    assert O.max_bin_err(ys, ref) <= REL_L2_TOL, f"{family} mode {mode}: max-bin {O.max_bin_err(ys, ref):.3e}"

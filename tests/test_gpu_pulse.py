"""Fused pulse compression on the GPU (sipFftMakePlanPulse1D).

Checks the fused chain against the FP64 oracle, against the plain
composition a reference user would write (asdFftExecC2C forward, an
elementwise multiply, asdFftExecC2C inverse), and through the batch work
queue alone and in a mix of lengths.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle
from tests.test_emu_pulse import signal

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-6
CASES = [(256, 64), (1000, 33), (4096, 16), (6000, 8), (15625, 3), (16384, 4), (20000, 3), (65536, 4),
         (1 << 18, 2)]


class Pulse:
    def __init__(self, torch, n, batch, flags, seed, generic=False):
        from sip_b200.fft import FftHandle, check

        self.n, self.batch, self.flags = n, batch, flags
        self.x = signal(n, batch, seed)
        self.filt = O.chirp_spectrum(n)
        self.xt = torch.from_numpy(self.x).cuda()
        self.ft = torch.from_numpy(self.filt.astype(np.complex64)).cuda()
        self.yt = torch.zeros_like(self.xt)
        self.h = FftHandle()
        if generic:
            check(self.h.set_hint(L.SIP_FFT_HINT_GENERIC_ONLY, 1), "hint")
        check(self.h.make_plan_pulse_1d(n, batch, self.ft.data_ptr(), flags), "sipFftMakePlanPulse1D")
        self.h.bind_workspace()

    def want(self):
        return O.pulse(self.x, self.filt, conj=bool(self.flags & 1), scale=bool(self.flags & 2))


@pytest.mark.parametrize("n,batch", CASES)
@pytest.mark.parametrize("flags", [1, 3])
def test_pulse_vs_fp64_and_plain_chain(cuda, n, batch, flags):
    from sip_b200.fft import FftHandle, check

    torch = cuda
    s = torch.cuda.Stream()
    p = Pulse(torch, n, batch, flags, 20261203 + n)
    check(p.h.set_stream(s), "stream")
    settle()
    check(p.h.exec_c2c(p.xt, p.yt), "asdFftExecC2C")
    s.synchronize()
    out = p.yt.cpu().numpy()
    assert O.rel_l2(out, p.want()) <= REL_L2_TOL
    # the plain composition: forward C2C, multiply, inverse C2C
    fwd, inv = FftHandle(), FftHandle()
    check(fwd.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, batch), "plan fwd")
    check(inv.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_INVERSE, batch), "plan inv")
    for h in (fwd, inv):
        h.bind_workspace()
        check(h.set_stream(s), "stream")
    spec = torch.empty_like(p.xt)
    y2 = torch.empty_like(p.xt)
    settle()
    check(fwd.exec_c2c(p.xt, spec), "fwd")
    with torch.cuda.stream(s):
        spec.mul_(p.ft.conj() if flags & 1 else p.ft)
    settle()
    check(inv.exec_c2c(spec, y2), "inv")
    s.synchronize()
    plain = y2.cpu().numpy() / (n if flags & 2 else 1)
    assert O.rel_l2(out, plain) <= 2 * REL_L2_TOL
    for h in (p.h, fwd, inv):
        h.destroy()


def test_pulse_in_place(cuda):
    from sip_b200.fft import check

    torch = cuda
    s = torch.cuda.Stream()
    for n in (4096, 65536):
        p = Pulse(torch, n, 3, 3, 7 + n)
        check(p.h.set_stream(s), "stream")
        settle()
        check(p.h.exec_raw(p.xt.data_ptr(), p.xt.data_ptr()), "exec in place")
        s.synchronize()
        assert O.rel_l2(p.xt.cpu().numpy(), p.want()) <= REL_L2_TOL
        p.h.destroy()


def test_pulse_batched_queue_mix_equals_alone(cuda):
    """Pulse plans of several lengths in one work-queue batch: each result is
    bitwise the result of its plan run alone through the queue, and within
    tolerance of the FP64 oracle."""
    from sip_b200.fft import Batch, check

    torch = cuda
    s = torch.cuda.Stream()
    ps = [Pulse(torch, n, b, 3, 99 + n, generic=True) for n, b in [(256, 40), (1000, 7), (4096, 5), (20000, 2),
                                                                      (65536, 1)]]
    with Batch(True) as bt:
        for p in ps:
            check(bt.add(p.h, p.xt.data_ptr(), p.yt.data_ptr()), "add")
        settle()
        check(bt.execute(s), "exec")
        s.synchronize()
        assert bt.take_status() == 0
    mixed = [p.yt.cpu().numpy() for p in ps]
    for p, m in zip(ps, mixed):
        assert O.rel_l2(m, p.want()) <= REL_L2_TOL
        p.yt.zero_()
        with Batch(True) as bt:
            check(bt.add(p.h, p.xt.data_ptr(), p.yt.data_ptr()), "add")
            settle()
            check(bt.execute(s), "exec")
            s.synchronize()
        np.testing.assert_array_equal(p.yt.cpu().numpy(), m)
        p.h.destroy()

"""sipFftExecC2CNoAlloc: C2C execution that allocates no device memory.

Callers such as a real-time signal chain (where a cudaMalloc or cudaFree
would synchronise the device and stall its other streams) or a host whose
GPU memory belongs to another pool cannot allocate a workspace while they
run.  This entry point runs the same kernels as the ordinary exec with the
plan's intermediate in the library's static 32 MiB device array.  The GPU
tests check it, through the C ABI, against the ordinary entry point
(sipFftExecRaw with a bound workspace) on two calls in a row, for every kind
of C2C plan that puts a pass in the workspace (four-step lengths, Bluestein
lengths above one tile, pulse compression above one tile, 2-D plans with the
output shift) and for an in-place call; and that the device's free memory
(cudaMemGetInfo) is the same before and after each call, the first one in
the process included.  This file is collected last so that a run stopping at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle, random_input

REL_L2_TOL = 1e-6

# (kind, sizes, direction, batch).  Every plan except the single-pass one
# needs scratch, each within the 32 MiB array.
CASES = [("four-step", [65536], O.FORWARD, 8), ("four-step", [32768], O.INVERSE, 16),
         ("single-pass", [4096], O.FORWARD, 4), ("bluestein", [20011], O.FORWARD, 3),
         ("pulse", [32768], O.FORWARD, 4), ("shift-2d", [96, 80], O.INVERSE, 3),
         ("in-place", [65536], O.INVERSE, 4)]


class Case:
    """Two identical plans: one run without workspace through the no-alloc
    entry point, one with a bound workspace through sipFftExecRaw."""

    def __init__(self, torch, kind, sizes, direction, batch, stream):
        from sip_b200.fft import FftHandle, check

        self.kind, self.sizes, self.direction, self.batch = kind, sizes, direction, batch
        self.filt = None
        if kind == "pulse":
            self.filt = torch.from_numpy(O.chirp_spectrum(sizes[0]).astype(np.complex64)).cuda()
        self.na, self.ref = FftHandle(), FftHandle()
        for h in (self.na, self.ref):
            if kind == "shift-2d":
                check(h.set_output_shift(1, 0.5), "sipFftSetOutputShift")
            if kind == "pulse":
                check(h.make_plan_pulse_1d(sizes[0], batch, self.filt.data_ptr(), 1), "sipFftMakePlanPulse1D")
            elif len(sizes) == 1:
                check(h.make_plan_1d(sizes[0], O.C2C, direction, batch), "asdFftMakePlan1D")
            else:
                check(h.make_plan_2d(sizes[0], sizes[1], O.C2C, direction, batch), "asdFftMakePlan2D")
            check(h.set_stream(stream), "asdFftSetStream")
        self.ref.bind_workspace()   # the no-alloc plan gets none

    def want(self, x):
        if self.kind == "pulse":
            return O.pulse(x, self.filt.cpu().numpy(), conj=True)
        y = O.fp64(O.C2C, self.direction, x, self.sizes)
        if self.kind == "shift-2d":  # fftshift of every output slice, times 0.5
            rows, cols = self.sizes
            g = O.shift2d(y.astype(np.complex128).reshape(-1), rows, cols, self.batch, 0, False)
            y = 0.5 * g.reshape(y.shape)
        return y

    def destroy(self):
        self.na.destroy()
        self.ref.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("kind,sizes,direction,batch", CASES)
def test_no_alloc_matches_ordinary_exec(cuda, kind, sizes, direction, batch):
    from sip_b200.fft import check

    torch = cuda
    lib = L.lib()
    s = torch.cuda.Stream()
    c = Case(torch, kind, sizes, direction, batch, s)
    for call in range(2):                            # two calls in a row
        x = random_input(O.C2C, sizes, batch, seed=7000 + call + sum(sizes))
        xt = torch.from_numpy(x).cuda()
        y_na = xt.clone() if kind == "in-place" else torch.zeros_like(xt)
        y_ref = torch.zeros_like(xt)
        src = y_na if kind == "in-place" else xt
        settle()
        free_before = torch.cuda.mem_get_info()[0]
        check(lib.sipFftExecC2CNoAlloc(c.na.h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(y_na.data_ptr())),
              "sipFftExecC2CNoAlloc")
        s.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {call}: device memory changed"
        check(c.ref.exec_raw(xt.data_ptr(), y_ref.data_ptr()), "sipFftExecRaw")
        s.synchronize()
        a, b = y_na.cpu().numpy(), y_ref.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), f"call {call}"
        assert O.rel_l2(a, c.want(x)) <= REL_L2_TOL, f"call {call}"
    c.destroy()


@pytest.mark.gpu
def test_no_alloc_rejects_oversized_and_non_c2c(cuda):
    from sip_b200.fft import FftHandle, check

    torch = cuda
    lib = L.lib()
    s = torch.cuda.Stream()
    n, batch = 65536, 128                           # 64 MiB intermediate > 32 MiB
    big = FftHandle()
    check(big.make_plan_1d(n, O.C2C, O.FORWARD, batch), "asdFftMakePlan1D")
    check(big.set_stream(s), "asdFftSetStream")
    x = torch.zeros(batch * n, dtype=torch.complex64, device="cuda")
    y = torch.zeros_like(x)
    settle()
    rc = lib.sipFftExecC2CNoAlloc(big.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
    assert rc == L.ACL_ERROR_INVALID_PARAM
    big.destroy()
    r2c = FftHandle()
    check(r2c.make_plan_1d(1000, O.R2C, O.FORWARD, 2), "plan")
    settle()
    rc = lib.sipFftExecC2CNoAlloc(r2c.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
    assert rc == L.ACL_ERROR_API_NOT_SUPPORT
    r2c.destroy()

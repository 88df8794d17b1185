"""sipFftExecC2CNoAlloc: C2C execution that allocates no device memory.

Callers such as a real-time signal chain (where a cudaMalloc or cudaFree
would synchronise the device and stall its other streams) or a host whose
GPU memory belongs to another pool cannot allocate a workspace while they
run.  This entry point runs the same kernels as the ordinary exec with the
two-pass intermediate in the library's static 32 MiB device array.  The
GPU test checks it, through the C ABI, against the ordinary entry point
(sipFftExecRaw with a bound workspace) on two calls in a row; the first
call in a fresh process also does the array's one-time set-up.  This file
is collected last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle, random_input

REL_L2_TOL = 1e-6

# (length, direction, batch): two-pass (four-step) lengths, whose plans need
# scratch, and one single-pass length.
CASES = [(65536, O.FORWARD, 8), (32768, O.INVERSE, 16), (4096, O.FORWARD, 4)]


def plan(lib, n, direction, batch, stream):
    from sip_b200.fft import FftHandle, check

    h = FftHandle()
    check(h.make_plan_1d(n, O.C2C, direction, batch), "asdFftMakePlan1D")
    check(h.set_stream(stream), "asdFftSetStream")
    return h


@pytest.mark.gpu
@pytest.mark.parametrize("n,direction,batch", CASES)
def test_no_alloc_matches_ordinary_exec(cuda, n, direction, batch):
    from sip_b200.fft import check

    torch = cuda
    lib = L.lib()
    s = torch.cuda.Stream()
    na = plan(lib, n, direction, batch, s)          # no workspace bound
    ref = plan(lib, n, direction, batch, s)
    ref.bind_workspace()
    for call in range(2):                            # two calls in a row
        x = random_input(O.C2C, [n], batch, seed=7000 + call)
        xt = torch.from_numpy(x).cuda()
        y_na = torch.zeros_like(xt)
        y_ref = torch.zeros_like(xt)
        settle()
        check(lib.sipFftExecC2CNoAlloc(na.h, ctypes.c_void_p(xt.data_ptr()), ctypes.c_void_p(y_na.data_ptr())),
              "sipFftExecC2CNoAlloc")
        settle()
        check(ref.exec_raw(xt.data_ptr(), y_ref.data_ptr()), "sipFftExecRaw")
        s.synchronize()
        a, b = y_na.cpu().numpy(), y_ref.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), f"call {call}"
        assert O.rel_l2(a, O.fp64(O.C2C, direction, x, [n])) <= REL_L2_TOL, f"call {call}"
    na.destroy()
    ref.destroy()


@pytest.mark.gpu
def test_no_alloc_rejects_oversized_and_non_c2c(cuda):
    torch = cuda
    lib = L.lib()
    s = torch.cuda.Stream()
    n, batch = 65536, 128                           # 64 MiB intermediate > 32 MiB
    big = plan(lib, n, O.FORWARD, batch, s)
    x = torch.zeros(batch * n, dtype=torch.complex64, device="cuda")
    y = torch.zeros_like(x)
    settle()
    rc = lib.sipFftExecC2CNoAlloc(big.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
    assert rc == L.ACL_ERROR_INVALID_PARAM
    big.destroy()
    from sip_b200.fft import FftHandle, check

    r2c = FftHandle()
    check(r2c.make_plan_1d(1000, O.R2C, O.FORWARD, 2), "plan")
    settle()
    rc = lib.sipFftExecC2CNoAlloc(r2c.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
    assert rc == L.ACL_ERROR_API_NOT_SUPPORT
    r2c.destroy()

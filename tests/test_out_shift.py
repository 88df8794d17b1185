"""fftshift / ifftshift fused into the C2C output store
(sipFftSetOutputShift): y = shift(FFT(x)) * scale for 1-D and 2-D plans,
against the oracle's FFT followed by the asdFftShift / asdIfftShift golden,
on the CPU harness and on the GPU."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import emu_run, random_input, settle

CASES = [([6], 3), ([7], 2), ([1000], 5), ([4096], 3), ([65536], 2), ([6, 8], 3), ([7, 9], 2), ([33, 65], 2),
         ([128, 50], 3), ([256, 256], 2)]


def want(x, sizes, direction, mode, scale):
    y = O.fp64(O.C2C, direction, x, sizes)
    b = x.shape[0]
    rows, cols = (1, sizes[0]) if len(sizes) == 1 else tuple(sizes)
    g = O.shift2d(y.astype(np.complex128).reshape(-1), rows, cols, b, 0, mode == 2)
    return g.astype(np.complex128).reshape(y.shape) * scale


@pytest.mark.parametrize("sizes,batch", CASES)
@pytest.mark.parametrize("mode,scale", [(1, 1.0), (2, 0.25)])
def test_out_shift_harness(emu, sizes, batch, mode, scale):
    emu.emu_set_out_shift.argtypes = [ctypes.c_int, ctypes.c_double]
    x = random_input(O.C2C, sizes, batch, seed=sum(sizes))
    emu.emu_set_out_shift(mode, scale)
    try:
        rc, out, desc = emu_run(emu, O.C2C, O.FORWARD, sizes, batch, x)
    finally:
        emu.emu_set_out_shift(0, 1.0)
    assert rc == 0, desc
    assert "shift" in desc
    assert O.rel_l2(out, want(x, sizes, O.FORWARD, mode, scale)) <= 1e-6


def test_out_shift_argument_checks(sip_lib):
    from sip_b200.fft import FftHandle

    h = FftHandle()
    assert h.set_output_shift(3) == L.ACL_ERROR_INVALID_PARAM
    assert h.set_output_shift(1) == L.ACL_SUCCESS
    assert h.make_plan_3d(8, 8, 8, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 1) == L.ACL_ERROR_INVALID_PARAM
    h.destroy()
    h = FftHandle()
    assert h.set_output_shift(1) == L.ACL_SUCCESS
    assert h.make_plan_1d(64, L.ASCEND_FFT_R2C, L.ASCEND_FFT_FORWARD, 1) == L.ACL_ERROR_INVALID_PARAM
    h.destroy()
    h = FftHandle()
    assert h.make_plan_1d(64, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 1) == L.ACL_SUCCESS
    assert h.set_output_shift(1) == L.ACL_ERROR_INVALID_PARAM  # after MakePlan
    h.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("sizes,batch", CASES + [([2048, 2048], 2), ([500, 50], 300)])
@pytest.mark.parametrize("mode,scale,direction", [(1, 1.0, O.FORWARD), (2, 1.0 / 64, O.INVERSE)])
def test_out_shift_gpu(cuda, sizes, batch, mode, scale, direction):
    from sip_b200.fft import FftHandle, check

    torch = cuda
    x = random_input(O.C2C, sizes, batch, seed=sum(sizes) + mode)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros_like(xt)
    h = FftHandle()
    check(h.set_output_shift(mode, scale), "shift")
    if len(sizes) == 1:
        check(h.make_plan_1d(sizes[0], O.C2C, direction, batch), "plan")
    else:
        check(h.make_plan_2d(sizes[0], sizes[1], O.C2C, direction, batch), "plan")
    h.bind_workspace()
    s = torch.cuda.Stream()
    check(h.set_stream(s), "stream")
    settle()
    check(h.exec_c2c(xt, yt), "exec")
    s.synchronize()
    assert O.rel_l2(yt.cpu().numpy(), want(x, sizes, direction, mode, scale)) <= 1e-6
    h.destroy()

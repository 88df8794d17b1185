"""asdFftExecC2CSeparated: C2C on separated real / imaginary float planes.
Argument checks of the reference (core/fft/fft_api.cpp:1912-1985) run
without a GPU; parity against the FP64 oracle runs on the GPU for the
reference's documented lengths 2..256 (FFT_1D.md) and beyond."""
import ctypes

import numpy as np
import pytest

from tests.fftcase import settle

from oracle import oracle as O
from sip_b200 import _lib as L
from sip_b200.fft import FftHandle, acl_tensor, check
from tests.test_shift import HostTensor

SEP = L.ASCEND_FFT_C2C_SEP


def test_separated_argument_checks(sip_lib):
    h = FftHandle()
    check(h.make_plan_1d(64, SEP, L.ASCEND_FFT_FORWARD, 4), "plan")
    f = [HostTensor([4, 64], L.ACL_FLOAT) for _ in range(4)]
    other = HostTensor([4, 32], L.ACL_FLOAT)
    c64 = HostTensor([4, 64], L.ACL_COMPLEX64)
    ex = sip_lib.asdFftExecC2CSeparated
    assert ex(None, f[0].h, f[1].h, f[2].h, f[3].h) == L.ACL_ERROR_INVALID_PARAM
    assert ex(h.h, f[0].h, other.h, f[2].h, f[3].h) == L.ACL_ERROR_INTERNAL_ERROR      # shapes differ
    assert ex(h.h, f[0].h, f[1].h, c64.h, f[3].h) == L.ACL_ERROR_OP_INPUT_NOT_MATCH    # not FLOAT
    wrong = [HostTensor([2, 64], L.ACL_FLOAT) for _ in range(4)]
    assert ex(h.h, *[t.h for t in wrong]) == L.ACL_ERROR_INVALID_PARAM                 # batch mismatch
    h.destroy()
    g = FftHandle()
    check(g.make_plan_1d(64, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 4), "plan")
    assert ex(g.h, f[0].h, f[1].h, f[2].h, f[3].h) == L.ACL_ERROR_INVALID_PARAM         # not a separated plan
    g.destroy()


def test_separated_plan_limits(sip_lib):
    h = FftHandle()
    assert h.make_plan_1d(1 << 16, SEP, L.ASCEND_FFT_FORWARD, 1) == L.ACL_ERROR_INVALID_PARAM  # beyond one tile
    h.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 7, 16, 100, 128, 243, 256, 1000, 4096])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
@pytest.mark.parametrize("in_place", [False, True])
def test_separated_parity(cuda, n, direction, in_place):
    torch = cuda
    batch = 37
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(np.complex64)
    re = torch.from_numpy(np.ascontiguousarray(x.real)).cuda()
    im = torch.from_numpy(np.ascontiguousarray(x.imag)).cuda()
    ore, oim = (re, im) if in_place else (torch.empty_like(re), torch.empty_like(im))
    h = FftHandle()
    check(h.make_plan_1d(n, SEP, direction, batch), "plan")
    s = torch.cuda.Stream()
    check(h.set_stream(s), "stream")
    with acl_tensor(re) as a, acl_tensor(im) as b, acl_tensor(ore) as c, acl_tensor(oim) as d:
        settle()
        check(L.lib().asdFftExecC2CSeparated(h.h, a, b, c, d), "exec separated")
    s.synchronize()
    out = ore.cpu().numpy() + 1j * oim.cpu().numpy()
    assert O.rel_l2(out, O.fp64(O.C2C, direction, x, [n])) <= 1e-6
    h.destroy()

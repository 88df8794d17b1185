"""asdFftShift / asdIfftShift: argument checks of the reference
(tests/ut/unittest/fft/fftshift/test_fftshift_negative.cpp) without a GPU,
and the reference's shift cases on the GPU against the numpy golden
(tests/ut/unittest/fft/fftshift/fftshift_data/gen_data.py)."""
import ctypes

import numpy as np
import pytest

from tests.fftcase import settle

from oracle import oracle as O
from sip_b200 import _lib as L
from sip_b200.fft import acl_tensor, create_acl_tensor

INV = L.ACL_ERROR_INVALID_PARAM

# (row, col, batch, dist): test_fftshift.cpp / test_ifftshift.cpp cases 0-9
CASES = [(6, 8, 3, 0), (7, 9, 2, 0), (1, 16, 4, 0), (16, 1, 2, 0), (4, 6, 3, 32), (33, 67, 5, 0), (128, 50, 6, 0),
         (64, 48, 8, 0), (500, 50, 12000, 0), (2, 10000, 2, 0)]
# ifftshift scale cases 10-14
SCALE_CASES = [(7, 9, 2, 0, 1.0 / 63.0), (500, 50, 12000, 0, 1.0 / 25000.0), (5, 8000, 2, 0, 0.25),
               (3, 10001, 2, 0, 0.5), (16, 1, 2, 0, -2.5)]


class HostTensor:
    """An aclTensor descriptor over host memory, for argument checks that
    must fail before anything touches the data."""

    def __init__(self, shape, dtype=L.ACL_COMPLEX64):
        self.buf = np.zeros(16, np.complex64)
        n = len(shape)
        dims = (ctypes.c_int64 * n)(*shape)
        st = (ctypes.c_int64 * n)(*([1] * n))
        self.h = L.lib().aclCreateTensor(dims, n, dtype, st, 0, L.ACL_FORMAT_ND, dims, n,
                                         ctypes.c_void_p(self.buf.ctypes.data))

    def __del__(self):
        L.lib().aclDestroyTensor(self.h)


def shift(lib, inverse, row, col, batch, dist, a, b, scale=1.0):
    if inverse:
        return lib.asdIfftShift(row, col, batch, dist, scale, a, b, None, None)
    return lib.asdFftShift(row, col, batch, dist, a, b, None, None)


@pytest.mark.parametrize("inverse", [False, True])
def test_rejected_arguments(sip_lib, inverse):
    t16 = HostTensor([16])
    big = 1 << 32
    assert shift(sip_lib, inverse, 0, 4, 1, 0, t16.h, t16.h) == INV
    assert shift(sip_lib, inverse, 4, -1, 1, 0, t16.h, t16.h) == INV
    assert shift(sip_lib, inverse, big, big, 1, 0, t16.h, t16.h) == INV              # row * col overflows
    assert shift(sip_lib, inverse, 1, 1, 1 << 32, 1 << 33, t16.h, t16.h) == INV    # (batch-1)*dist overflows
    assert shift(sip_lib, inverse, 2, 2, 4, 3, t16.h, t16.h) == INV                # 0 < dist < row*col
    wrapped = HostTensor([(1 << 40) + 1, 1 << 24])                                 # element count wraps
    assert shift(sip_lib, inverse, 1000, 1000, 1, 0, wrapped.h, t16.h) == INV
    assert shift(sip_lib, inverse, 2, 2, 4, 0, t16.h, wrapped.h) == INV
    assert shift(sip_lib, inverse, 2, 2, 8, 0, t16.h, HostTensor([16]).h) == INV   # 32 elements needed
    f32 = HostTensor([16], L.ACL_FLOAT)
    assert shift(sip_lib, inverse, 2, 2, 1, 0, f32.h, t16.h) == L.ACL_ERROR_UNSUPPORTED_DATA_TYPE
    assert shift(sip_lib, inverse, 2, 2, 4, 0, t16.h, t16.h) == INV                # input and output overlap


def test_golden_matches_numpy_even_sizes():
    x = (np.arange(48) + 1j * np.arange(48)).astype(np.complex64)
    g = O.shift2d(x, 6, 8, 1, 0, inverse=False)
    np.testing.assert_array_equal(g[0], np.fft.fftshift(x.reshape(6, 8)))
    gi = O.shift2d(x, 6, 8, 1, 0, inverse=True)
    np.testing.assert_array_equal(gi[0], np.fft.ifftshift(x.reshape(6, 8)))


def _run_gpu(torch, row, col, batch, dist, inverse, scale=1.0):
    rng = np.random.default_rng(row * 7 + col)
    d = dist if dist > 0 else row * col
    n_in = (batch - 1) * d + row * col
    x = (rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)).astype(np.complex64)
    xt = torch.from_numpy(x).cuda()
    yt = torch.zeros((batch, row, col), dtype=torch.complex64, device="cuda")
    s = torch.cuda.Stream()
    lib = L.lib()
    with acl_tensor(xt, [n_in]) as a, acl_tensor(yt) as b:
        if inverse:
            settle()
            rc = lib.asdIfftShift(row, col, batch, dist, scale, a, b, ctypes.c_void_p(s.cuda_stream), None)
        else:
            settle()
            rc = lib.asdFftShift(row, col, batch, dist, a, b, ctypes.c_void_p(s.cuda_stream), None)
    assert rc == L.ACL_SUCCESS
    s.synchronize()
    return yt.cpu().numpy(), O.shift2d(x, row, col, batch, dist, inverse, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("row,col,batch,dist", CASES)
def test_shift_cases(cuda, inverse, row, col, batch, dist):
    out, want = _run_gpu(cuda, row, col, batch, dist, inverse)
    np.testing.assert_array_equal(out, want)          # a permutation: bit exact


@pytest.mark.gpu
@pytest.mark.parametrize("row,col,batch,dist,scale", SCALE_CASES)
def test_ifftshift_scale_cases(cuda, row, col, batch, dist, scale):
    out, want = _run_gpu(cuda, row, col, batch, dist, True, scale)
    np.testing.assert_array_equal(out, want)          # one float32 multiply per component

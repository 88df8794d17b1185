"""PyTorch binding (sip_b200.torch_sip), the sip_pta mirror: op registration
and the LRU plan cache on the CPU; every op against the FP64 oracle on the
GPU."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from sip_b200 import _lib as L
from sip_b200 import torch_sip as ts


def test_ops_registered():
    for name in ("asd_fft_c2c", "asd_fft_r2c", "asd_fft_c2r", "asd_fft_c2c_sep"):
        assert hasattr(torch.ops.torch_sip, name)


def test_lru_cache_evicts_oldest():
    cache = ts.FFTMixCache(3)
    keys = [((64 * (i + 1),), L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 2) for i in range(4)]
    hs = [cache.get(k, "cpu") for k in keys[:3]]
    assert cache.get(keys[0], "cpu") is hs[0]          # hit moves keys[0] to the back
    cache.get(keys[3], "cpu")                          # evicts keys[1], the least recent
    assert cache.size() == 3 and keys[1] not in cache.entries and keys[0] in cache.entries
    assert hs[1].h is None                             # evicted handles are destroyed
    cache.set_capacity(1)
    assert list(cache.entries) == [keys[3]]
    cache.clear()
    assert cache.size() == 0
    assert ts.DEFAULT_CACHE_SIZE == 10 and ts.CACHE.capacity == 10


def test_input_checks():
    with pytest.raises(ValueError):
        ts.asd_fft_c2c(torch.zeros(4, 8, dtype=torch.complex64))   # not a CUDA tensor


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(3, 1000), (2, 64, 48), (1, 16, 32, 20)])
@pytest.mark.parametrize("fwd", [True, False])
def test_c2c_r2c_c2r(cuda, shape, fwd):
    rng = np.random.default_rng(len(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    d = O.FORWARD if fwd else O.INVERSE
    y = ts.asd_fft_c2c(torch.from_numpy(x).cuda(), fwd).cpu().numpy()
    assert O.rel_l2(y, O.fp64(O.C2C, d, x, shape[1:])) <= 1e-6
    xr = rng.uniform(-1, 1, shape).astype(np.float32)
    yr = torch.ops.torch_sip.asd_fft_r2c(torch.from_numpy(xr).cuda(), fwd).cpu().numpy()
    assert O.rel_l2(yr, O.fp64(O.R2C, d, xr, shape[1:])) <= 1e-6
    spec = O.fp64(O.R2C, O.FORWARD, xr, shape[1:]).astype(np.complex64)
    back = ts.asd_fft_c2r(torch.from_numpy(spec).cuda(), fwd).cpu().numpy()
    assert back.shape == shape
    assert O.rel_l2(back, O.fp64(O.C2R, d, spec, shape[1:])) <= 1e-6


@pytest.mark.gpu
def test_sep_and_shift_ops(cuda):
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((5, 256)) + 1j * rng.standard_normal((5, 256))).astype(np.complex64)
    re, im = ts.asd_fft_c2c_sep(torch.from_numpy(x.real.copy()).cuda(), torch.from_numpy(x.imag.copy()).cuda())
    out = re.cpu().numpy() + 1j * im.cpu().numpy()
    assert O.rel_l2(out, O.fp64(O.C2C, O.FORWARD, x, [256])) <= 1e-6
    s = (rng.standard_normal((4, 7, 9)) + 1j * rng.standard_normal((4, 7, 9))).astype(np.complex64)
    st = torch.from_numpy(s).cuda()
    np.testing.assert_array_equal(ts.fft_shift(st).cpu().numpy(), O.shift2d(s.reshape(-1), 7, 9, 4, 0, False))
    np.testing.assert_array_equal(ts.ifft_shift(st, scale=0.5).cpu().numpy(),
                                  O.shift2d(s.reshape(-1), 7, 9, 4, 0, True, 0.5))


@pytest.mark.gpu
def test_cache_reuse_and_eviction_on_gpu(cuda):
    ts.CACHE.clear()
    x = torch.randn(4, 4096, dtype=torch.complex64, device="cuda")
    a = ts.asd_fft_c2c(x)
    b = ts.asd_fft_c2c(x)
    assert ts.CACHE.size() == 1 and torch.equal(a, b)
    for n in range(1, 12):
        ts.asd_fft_c2c(torch.randn(2, 64 * n, dtype=torch.complex64, device="cuda"))
    assert ts.CACHE.size() == 10
    ts.CACHE.clear()

"""PyTorch binding of the FFT library, mirroring the reference's sip_pta
(sip_pta/torch_sip/__init__.py:427-447, csrc/fft/asd_fft_*.cpp,
csrc/FFTMixCache.*) on CUDA tensors.

Ops are registered as ``torch.ops.torch_sip.*`` and exposed as functions of
the same names:

* ``asd_fft_c2c(x, is_forward)``: complex64 [batch, X(, Y(, Z))] -> same shape
* ``asd_fft_r2c(x, is_forward)``: float32 -> complex64, last dim n // 2 + 1
* ``asd_fft_c2r(x, is_forward)``: complex64 -> float32, last dim 2 * (m - 1)
* ``asd_fft_c2c_sep(re, im, is_forward)``: separated float planes, 1-D
* ``fft_shift(x, row, col, batch, dist)`` / ``ifft_shift(..., scale)``

As in sip_pta, the leading dimension is the batch and the remaining 1-3
dimensions are the transform; plans live in an LRU cache of 10 entries
keyed by (sizes, type, direction, batch) (FFTMixCache DEFAULT_CACHE_SIZE),
each with its workspace kept resident on the device, and every call runs on
the current CUDA stream.  Inputs that are not contiguous are made so.
"""
from __future__ import annotations

import collections
import threading

import torch

from . import _lib as L
from .fft import FftHandle, FftError, acl_tensor, check

DEFAULT_CACHE_SIZE = 10


class FFTMixCache:
    """LRU cache of planned handles (sip_pta csrc/FFTMixCache.cpp)."""

    def __init__(self, capacity: int = DEFAULT_CACHE_SIZE):
        self.capacity = capacity
        self.entries: collections.OrderedDict = collections.OrderedDict()
        self.lock = threading.Lock()

    def get(self, key, device) -> FftHandle:
        with self.lock:
            if key in self.entries:
                self.entries.move_to_end(key)
                return self.entries[key]
            sizes, fft_type, direction, batch = key
            h = FftHandle()
            if len(sizes) == 1:
                rc = h.make_plan_1d(sizes[0], fft_type, direction, batch)
            elif len(sizes) == 2:
                rc = h.make_plan_2d(sizes[0], sizes[1], fft_type, direction, batch)
            else:
                rc = h.make_plan_3d(sizes[0], sizes[1], sizes[2], fft_type, direction, batch)
            if rc != L.ACL_SUCCESS:
                h.destroy()
                raise FftError(f"make plan {key}", rc)
            h.bind_workspace(device)  # resident with the cache entry
            self.entries[key] = h
            while len(self.entries) > max(self.capacity, 0):
                _, old = self.entries.popitem(last=False)
                old.destroy()
            return h

    def set_capacity(self, capacity: int) -> None:
        with self.lock:
            self.capacity = capacity
            while len(self.entries) > max(capacity, 0):
                _, old = self.entries.popitem(last=False)
                old.destroy()

    def size(self) -> int:
        return len(self.entries)

    def clear(self) -> None:
        with self.lock:
            for h in self.entries.values():
                h.destroy()
            self.entries.clear()


CACHE = FFTMixCache()


def _direction(is_forward: bool) -> int:
    return L.ASCEND_FFT_FORWARD if is_forward else L.ASCEND_FFT_INVERSE


def _check_input(x: torch.Tensor, dtype, name: str) -> torch.Tensor:
    if not x.is_cuda:
        raise ValueError(f"{name}: input must be a CUDA tensor")
    if x.dtype != dtype:
        raise TypeError(f"{name}: input must be {dtype}, got {x.dtype}")
    if not 2 <= x.dim() <= 4:
        raise ValueError(f"{name}: input tensor must have 2, 3 or 4 dimensions, but got {x.dim()}")
    return x.contiguous()


# cudaStreamLegacy: the handle of the legacy default stream, passed when
# torch's current stream is the default one (the C ABI, like the reference,
# rejects a null stream).
_LEGACY_STREAM = 1


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream or _LEGACY_STREAM


def _run(key, fn_name: str, x: torch.Tensor, y: torch.Tensor) -> None:
    h = CACHE.get(key, x.device)
    check(h.set_stream(_stream(x.device)), "asdFftSetStream")
    fn = getattr(h.lib, fn_name)
    with acl_tensor(x) as a, acl_tensor(y) as b:
        check(fn(h.h, a, b), fn_name)


@torch.library.custom_op("torch_sip::asd_fft_c2c", mutates_args=())
def asd_fft_c2c(input_tensor: torch.Tensor, is_forward: bool = True) -> torch.Tensor:
    x = _check_input(input_tensor, torch.complex64, "asd_fft_c2c")
    y = torch.empty_like(x)
    _run((tuple(x.shape[1:]), L.ASCEND_FFT_C2C, _direction(is_forward), x.shape[0]), "asdFftExecC2C", x, y)
    return y


@torch.library.custom_op("torch_sip::asd_fft_r2c", mutates_args=())
def asd_fft_r2c(input_tensor: torch.Tensor, is_forward: bool = True) -> torch.Tensor:
    x = _check_input(input_tensor, torch.float32, "asd_fft_r2c")
    shape = list(x.shape)
    shape[-1] = shape[-1] // 2 + 1
    y = torch.empty(shape, dtype=torch.complex64, device=x.device)
    _run((tuple(x.shape[1:]), L.ASCEND_FFT_R2C, _direction(is_forward), x.shape[0]), "asdFftExecR2C", x, y)
    return y


@torch.library.custom_op("torch_sip::asd_fft_c2r", mutates_args=())
def asd_fft_c2r(input_tensor: torch.Tensor, is_forward: bool = True) -> torch.Tensor:
    x = _check_input(input_tensor, torch.complex64, "asd_fft_c2r")
    shape = list(x.shape)
    shape[-1] = (shape[-1] - 1) * 2
    y = torch.empty(shape, dtype=torch.float32, device=x.device)
    _run((tuple(shape[1:]), L.ASCEND_FFT_C2R, _direction(is_forward), x.shape[0]), "asdFftExecC2R", x, y)
    return y


@torch.library.custom_op("torch_sip::asd_fft_c2c_sep", mutates_args=())
def asd_fft_c2c_sep(in_real: torch.Tensor, in_imag: torch.Tensor,
                    is_forward: bool = True) -> tuple[torch.Tensor, torch.Tensor]:
    re = _check_input(in_real, torch.float32, "asd_fft_c2c_sep")
    im = _check_input(in_imag, torch.float32, "asd_fft_c2c_sep")
    if re.shape != im.shape:
        raise ValueError("asd_fft_c2c_sep: real and imaginary planes differ in shape")
    if re.dim() != 2:
        raise ValueError("asd_fft_c2c_sep: separated planes are 1-D transforms [batch, n]")
    ore, oim = torch.empty_like(re), torch.empty_like(im)
    h = CACHE.get(((re.shape[1],), L.ASCEND_FFT_C2C_SEP, _direction(is_forward), re.shape[0]), re.device)
    check(h.set_stream(_stream(re.device)), "asdFftSetStream")
    with acl_tensor(re) as a, acl_tensor(im) as b, acl_tensor(ore) as c, acl_tensor(oim) as d:
        check(h.lib.asdFftExecC2CSeparated(h.h, a, b, c, d), "asdFftExecC2CSeparated")
    return ore, oim


def _shift_dims(x: torch.Tensor, row, col, batch, dist):
    if row is None or col is None or batch is None:
        if x.dim() != 3:
            raise ValueError("fft_shift: give row, col and batch for inputs that are not [batch, row, col]")
        batch, row, col = x.shape
    return int(row), int(col), int(batch), int(dist)


def _shift(x: torch.Tensor, row, col, batch, dist, inverse: bool, scale: float) -> torch.Tensor:
    if not x.is_cuda or x.dtype != torch.complex64:
        raise TypeError("fft_shift: input must be a complex64 CUDA tensor")
    row, col, batch, dist = _shift_dims(x, row, col, batch, dist)
    x = x.contiguous()
    y = torch.empty((batch, row, col), dtype=torch.complex64, device=x.device)
    lib = L.lib()
    stream = _stream(x.device)
    import ctypes

    with acl_tensor(x, [x.numel()]) as a, acl_tensor(y) as b:
        if inverse:
            rc = lib.asdIfftShift(row, col, batch, dist, scale, a, b, ctypes.c_void_p(stream), None)
        else:
            rc = lib.asdFftShift(row, col, batch, dist, a, b, ctypes.c_void_p(stream), None)
    check(rc, "asdIfftShift" if inverse else "asdFftShift")
    return y


def fft_shift(input_tensor: torch.Tensor, row: int | None = None, col: int | None = None, batch: int | None = None,
              dist: int = 0) -> torch.Tensor:
    """output[s][(r + (row+1)//2) % row][(c + (col+1)//2) % col] = input[s][r][c]."""
    return _shift(input_tensor, row, col, batch, dist, False, 1.0)


def ifft_shift(input_tensor: torch.Tensor, row: int | None = None, col: int | None = None, batch: int | None = None,
               dist: int = 0, scale: float = 1.0) -> torch.Tensor:
    """output[s][(r + row//2) % row][(c + col//2) % col] = scale * input[s][r][c]."""
    return _shift(input_tensor, row, col, batch, dist, True, scale)

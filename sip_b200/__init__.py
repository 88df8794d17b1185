"""B200-native FFT library behind the hicann/sip ``fft_api.h`` C ABI.

The product is the in-tree shared library ``libsip_fft.so`` (CUDA kernels
for sm_100a + C++ planner).  This package holds its build recipe
(``build.py``), a ctypes binding (``_lib``) and a host-side mirror of the
reference's plan/exec interface (``fft``).
"""
from . import _lib
from .fft import FftHandle, FftError, acl_tensor, check

__all__ = ["FftHandle", "FftError", "acl_tensor", "check", "_lib"]

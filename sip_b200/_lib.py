"""ctypes binding of the library's C ABI (include/fft_api.h,
include/sip_fft_ext.h, include/acl_tensor.h).

The shared library is built in-tree by ``sip_b200/build.py``.  Loading
fails loudly when it is missing: there is no other implementation.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsip_fft.so"

# Status codes (include/utils/aspb_status.h).
ACL_SUCCESS = 0
ACL_ERROR_INVALID_PARAM = 100000
ACL_ERROR_OP_INPUT_NOT_MATCH = 100021
ACL_ERROR_OP_OUTPUT_NOT_MATCH = 100022
ACL_ERROR_UNSUPPORTED_DATA_TYPE = 100026
ACL_ERROR_API_NOT_SUPPORT = 200001
ACL_ERROR_INTERNAL_ERROR = 500000

# asdFftType / asdFftDirection / asdFft1dDimType (include/fft_api.h).
ASCEND_FFT_C2C = 0x10
ASCEND_FFT_C2R = 0x11
ASCEND_FFT_R2C = 0x12
ASCEND_STFT_C2C = 0x20
ASCEND_STFT_C2R = 0x21
ASCEND_STFT_R2C = 0x22
ASCEND_FFT_C2C_SEP = 0x30
ASCEND_FFT_FORWARD = 0x10
ASCEND_FFT_INVERSE = 0x11
ASCEND_FFT_HORIZONTAL = 0x10
ASCEND_FFT_VERTICAL = 0x11

# Compute forms (include/sip_fft_ext.h).
SIP_FFT_COMPUTE_FP32 = 0
SIP_FFT_COMPUTE_TC_SPLIT = 1

# Planner hint keys (include/sip_fft_ext.h).
SIP_FFT_HINT_TILE_TRANSFORMS = 1
SIP_FFT_HINT_ELEMS_PER_THREAD = 2
SIP_FFT_HINT_GENERIC_ONLY = 3
SIP_FFT_HINT_RADIX_ORDER = 4
SIP_FFT_HINT_REAL_FUSED = 5
SIP_FFT_HINT_SK_VARIANT = 6
SIP_FFT_HINT_RUNTIME_COMPILE = 7

# Output shift modes (sipFftSetOutputShift).
SIP_FFT_SHIFT_NONE = 0
SIP_FFT_SHIFT_FFTSHIFT = 1
SIP_FFT_SHIFT_IFFTSHIFT = 2

# Pulse-compression flags.
SIP_FFT_PULSE_CONJ_FILTER = 1
SIP_FFT_PULSE_SCALE = 2

# Batch status bits.
SIP_FFT_BATCH_GATE_TIMEOUT = 2

# aclDataType / aclFormat (include/acl_tensor.h).
ACL_FLOAT = 0
ACL_COMPLEX64 = 16
ACL_FORMAT_ND = 2

# Every symbol the headers declare; tests check the library exports them.
EXPORTED = [
    "asdFftCreate", "asdFftSetStream", "asdFftMakePlan1D", "asdFftIstftMakePlan", "asdFftExecC2C",
    "asdFftExecC2CSeparated", "asdFftExecC2R", "asdFftExecR2C", "asdFftExecIstft", "asdFftDestroy",
    "asdFftMakePlan2D", "asdFftMakePlan3D", "asdFftGetWorkspaceSize", "asdFftSetWorkspace",
    "asdFftSynchronize", "asdFftGetType", "asdFftShift", "asdIfftShift",
    "sipFftExecRaw", "sipFftDescribePlan", "sipFftVersion", "sipFftSetComputeMode", "sipFftTakeDeviceErrors",
    "sipFftSetPlanHint", "sipFftBatchCreate", "sipFftBatchDestroy", "sipFftBatchClear", "sipFftBatchAdd",
    "sipFftBatchExec", "sipFftBatchSetGate", "sipFftBatchUseGraphs", "sipFftBatchTakeStatus",
    "sipFftExecC2CNoAlloc", "sipFftMakePlanPulse1D", "sipFftBatchAddRows", "sipFftSetOutputShift",
    "sipFftJitCompileCheck", "sipFftJitWait", "sipFftExecRawRows",
    "aclCreateTensor", "aclDestroyTensor", "aclGetViewShape", "aclGetDataType", "aclFreeViewShape",
    "aclGetTensorData",
]

_lib: ctypes.CDLL | None = None

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


def _declare(lib: ctypes.CDLL) -> None:
    sig = {
        "asdFftCreate": (_i32, [ctypes.POINTER(_vp)]),
        "asdFftSetStream": (_i32, [_vp, _vp]),
        "asdFftMakePlan1D": (_i32, [_vp, _i64, ctypes.c_int, ctypes.c_int, _i64, ctypes.c_int]),
        "asdFftMakePlan2D": (_i32, [_vp, _i64, _i64, ctypes.c_int, ctypes.c_int, _i32]),
        "asdFftMakePlan3D": (_i32, [_vp, _i64, _i64, _i64, ctypes.c_int, ctypes.c_int, _i32]),
        "asdFftExecC2C": (_i32, [_vp, _vp, _vp]),
        "asdFftExecC2R": (_i32, [_vp, _vp, _vp]),
        "asdFftExecR2C": (_i32, [_vp, _vp, _vp]),
        "asdFftExecC2CSeparated": (_i32, [_vp, _vp, _vp, _vp, _vp]),
        "asdFftDestroy": (_i32, [_vp]),
        "asdFftGetWorkspaceSize": (_i32, [_vp, ctypes.POINTER(ctypes.c_size_t)]),
        "asdFftSetWorkspace": (_i32, [_vp, _vp]),
        "asdFftSynchronize": (_i32, [_vp]),
        "asdFftGetType": (_i32, [_vp, ctypes.POINTER(ctypes.c_int)]),
        "asdFftShift": (_i32, [_i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
        "asdIfftShift": (_i32, [_i64, _i64, _i64, _i64, ctypes.c_double, _vp, _vp, _vp, _vp]),
        "sipFftExecRaw": (_i32, [_vp, _vp, _vp]),
        "sipFftExecRawRows": (_i32, [_vp, ctypes.c_longlong, _vp, _vp, _vp]),
        "sipFftDescribePlan": (_i32, [_vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
        "sipFftVersion": (ctypes.c_char_p, []),
        "sipFftSetComputeMode": (_i32, [_vp, ctypes.c_int]),
        "sipFftTakeDeviceErrors": (_i32, [ctypes.POINTER(ctypes.c_uint)]),
        "sipFftSetPlanHint": (_i32, [_vp, ctypes.c_int, ctypes.c_int]),
        "sipFftBatchCreate": (_i32, [ctypes.POINTER(_vp)]),
        "sipFftBatchDestroy": (_i32, [_vp]),
        "sipFftBatchClear": (_i32, [_vp]),
        "sipFftBatchAdd": (_i32, [_vp, _vp, _vp, _vp]),
        "sipFftBatchExec": (_i32, [_vp, _vp]),
        "sipFftBatchSetGate": (_i32, [_vp, _vp, ctypes.c_longlong]),
        "sipFftBatchUseGraphs": (_i32, [_vp, ctypes.c_int]),
        "sipFftBatchTakeStatus": (_i32, [_vp, ctypes.POINTER(ctypes.c_uint)]),
        "sipFftExecC2CNoAlloc": (_i32, [_vp, _vp, _vp]),
        "sipFftJitCompileCheck": (_i32, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_longlong]),
        "sipFftJitWait": (_i32, [ctypes.c_longlong]),
        "sipFftMakePlanPulse1D": (_i32, [_vp, _i64, _i64, _vp, ctypes.c_int]),
        "sipFftBatchAddRows": (_i32, [_vp, _vp, _vp, _vp, _i64, _vp]),
        "sipFftSetOutputShift": (_i32, [_vp, ctypes.c_int, ctypes.c_double]),
        "aclCreateTensor": (_vp, [ctypes.POINTER(_i64), ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_i64), _i64,
                                  ctypes.c_int, ctypes.POINTER(_i64), ctypes.c_uint64, _vp]),
        "aclDestroyTensor": (ctypes.c_int, [_vp]),
        "aclGetViewShape": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.POINTER(_i64)), ctypes.POINTER(ctypes.c_uint64)]),
        "aclGetDataType": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
        "aclFreeViewShape": (None, [ctypes.POINTER(_i64)]),
        "aclGetTensorData": (_vp, [_vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m sip_b200.build` (or __graft_entry__.build())")
        l = ctypes.CDLL(str(LIB_PATH))
        _declare(l)
        _lib = l
    return _lib

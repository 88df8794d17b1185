"""Python host mirror of the FFT C ABI.

`FftHandle` wraps one ``asdFftHandle`` and follows the reference's call
order (example/A2/FFT/1d/example_acl_fft_c2c_1d.cpp of hicann/sip):
create -> make plan -> get/set workspace -> set stream -> exec ->
synchronize -> destroy.  Tensors are torch CUDA tensors, described to the
library through the aclTensor shim (include/acl_tensor.h).  Every status
code is returned unchanged; `check` raises on non-zero.
"""
from __future__ import annotations

import ctypes
import json
from contextlib import contextmanager

from . import _lib as L


class FftError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} returned {code}")
        self.code = code


def check(code: int, what: str = "call") -> None:
    if code != L.ACL_SUCCESS:
        raise FftError(what, code)


def _dtype_code(t) -> int:
    import torch

    if t.dtype == torch.complex64:
        return L.ACL_COMPLEX64
    if t.dtype == torch.float32:
        return L.ACL_FLOAT
    raise TypeError(f"unsupported dtype {t.dtype}")


def create_acl_tensor(t, shape=None, dtype_code=None) -> int:
    """aclCreateTensor over a torch tensor's storage (view shape defaults to
    the tensor's shape)."""
    shape = list(t.shape if shape is None else shape)
    n = len(shape)
    dims = (ctypes.c_int64 * max(n, 1))(*shape)
    strides = [1] * n
    for i in range(n - 2, -1, -1):
        strides[i] = strides[i + 1] * shape[i + 1]
    st = (ctypes.c_int64 * max(n, 1))(*strides)
    code = _dtype_code(t) if dtype_code is None else dtype_code
    h = L.lib().aclCreateTensor(dims, n, code, st, 0, L.ACL_FORMAT_ND, dims, n, ctypes.c_void_p(t.data_ptr()))
    if not h:
        raise RuntimeError("aclCreateTensor failed")
    return h


@contextmanager
def acl_tensor(t, shape=None, dtype_code=None):
    h = create_acl_tensor(t, shape, dtype_code)
    try:
        yield h
    finally:
        L.lib().aclDestroyTensor(h)


class FftHandle:
    """One plan handle of the C ABI."""

    def __init__(self):
        self.lib = L.lib()
        h = ctypes.c_void_p()
        check(self.lib.asdFftCreate(ctypes.byref(h)), "asdFftCreate")
        self.h = h
        self.workspace = None  # torch tensor owning the bound workspace

    # ------------------------------------------------------------ plans
    def set_compute_mode(self, mode: int) -> int:
        return self.lib.sipFftSetComputeMode(self.h, mode)

    def set_hint(self, key: int, value: int) -> int:
        return self.lib.sipFftSetPlanHint(self.h, key, value)

    def make_plan_1d(self, n, fft_type, direction, batch, dim_type=L.ASCEND_FFT_HORIZONTAL) -> int:
        return self.lib.asdFftMakePlan1D(self.h, n, fft_type, direction, batch, dim_type)

    def set_output_shift(self, mode: int, scale: float = 1.0) -> int:
        """sipFftSetOutputShift: fftshift (1) / ifftshift (2) fused into the output store."""
        return self.lib.sipFftSetOutputShift(self.h, mode, scale)

    def make_plan_pulse_1d(self, n, batch, filter_ptr: int, flags: int = 0) -> int:
        """sipFftMakePlanPulse1D: y = IFFT(FFT(x) * F) per row; F lives on the
        device at filter_ptr (n complex64 values) and must outlive the plan."""
        return self.lib.sipFftMakePlanPulse1D(self.h, n, batch, ctypes.c_void_p(filter_ptr), flags)

    def make_plan_2d(self, x, y, fft_type, direction, batch) -> int:
        return self.lib.asdFftMakePlan2D(self.h, x, y, fft_type, direction, batch)

    def make_plan_3d(self, x, y, z, fft_type, direction, batch) -> int:
        return self.lib.asdFftMakePlan3D(self.h, x, y, z, fft_type, direction, batch)

    def workspace_size(self) -> tuple[int, int]:
        sz = ctypes.c_size_t(0)
        rc = self.lib.asdFftGetWorkspaceSize(self.h, ctypes.byref(sz))
        return rc, sz.value

    def set_workspace_ptr(self, ptr: int) -> int:
        return self.lib.asdFftSetWorkspace(self.h, ctypes.c_void_p(ptr))

    def bind_workspace(self, device=None) -> int:
        """GetWorkspaceSize, allocate it with torch and bind it (no-op when 0)."""
        import torch

        rc, size = self.workspace_size()
        check(rc, "asdFftGetWorkspaceSize")
        if size > 0:
            self.workspace = torch.empty(size, dtype=torch.uint8, device=device or "cuda")
            check(self.set_workspace_ptr(self.workspace.data_ptr()), "asdFftSetWorkspace")
        return size

    def set_stream(self, stream) -> int:
        """stream: torch.cuda.Stream, raw cudaStream_t int, or None (rejected)."""
        ptr = getattr(stream, "cuda_stream", stream)
        return self.lib.asdFftSetStream(self.h, ctypes.c_void_p(ptr) if ptr else None)

    # ------------------------------------------------------------- exec
    def exec_c2c(self, x, y, in_shape=None, out_shape=None) -> int:
        with acl_tensor(x, in_shape) as a, acl_tensor(y, out_shape) as b:
            return self.lib.asdFftExecC2C(self.h, a, b)

    def exec_r2c(self, x, y, in_shape=None, out_shape=None) -> int:
        with acl_tensor(x, in_shape) as a, acl_tensor(y, out_shape) as b:
            return self.lib.asdFftExecR2C(self.h, a, b)

    def exec_c2r(self, x, y, in_shape=None, out_shape=None) -> int:
        with acl_tensor(x, in_shape) as a, acl_tensor(y, out_shape) as b:
            return self.lib.asdFftExecC2R(self.h, a, b)

    def exec_raw(self, in_ptr: int, out_ptr: int) -> int:
        return self.lib.sipFftExecRaw(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr))

    def exec_rows(self, rows: int, in_ptr: int, out_ptr: int, ws_ptr: int | None = None) -> int:
        """The plan on its first `rows` transforms (sipFftExecRawRows)."""
        return self.lib.sipFftExecRawRows(self.h, ctypes.c_longlong(rows), ctypes.c_void_p(in_ptr),
                                          ctypes.c_void_p(out_ptr), ctypes.c_void_p(ws_ptr or 0))

    def synchronize(self) -> int:
        return self.lib.asdFftSynchronize(self.h)

    def get_type(self) -> tuple[int, int]:
        t = ctypes.c_int(0)
        rc = self.lib.asdFftGetType(self.h, ctypes.byref(t))
        return rc, t.value

    def describe(self) -> dict:
        need = ctypes.c_size_t(0)
        check(self.lib.sipFftDescribePlan(self.h, None, 0, ctypes.byref(need)), "sipFftDescribePlan")
        buf = ctypes.create_string_buffer(need.value)
        check(self.lib.sipFftDescribePlan(self.h, buf, need.value, ctypes.byref(need)), "sipFftDescribePlan")
        return json.loads(buf.value.decode())

    def destroy(self) -> int:
        rc = L.ACL_SUCCESS
        if self.h is not None:
            rc = self.lib.asdFftDestroy(self.h)
            self.h = None
        self.workspace = None
        return rc

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """Batched execution of many planned handles (sipFftBatch*): pass k of
    every added plan runs in one persistent work-queue launch, replayed from
    a captured CUDA graph when the wave structure repeats."""

    def __init__(self, use_graphs: bool = True):
        self.lib = L.lib()
        b = ctypes.c_void_p()
        check(self.lib.sipFftBatchCreate(ctypes.byref(b)), "sipFftBatchCreate")
        self.b = b
        check(self.lib.sipFftBatchUseGraphs(self.b, int(use_graphs)), "sipFftBatchUseGraphs")

    def add(self, handle: FftHandle, in_ptr: int, out_ptr: int) -> int:
        return self.lib.sipFftBatchAdd(self.b, handle.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr))

    def add_rows(self, handle: FftHandle, in_ptr: int, out_ptr: int, rows: int, ws_ptr: int | None = None) -> int:
        return self.lib.sipFftBatchAddRows(self.b, handle.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), rows,
                                           ctypes.c_void_p(ws_ptr) if ws_ptr else None)

    def execute(self, stream) -> int:
        ptr = getattr(stream, "cuda_stream", stream)
        return self.lib.sipFftBatchExec(self.b, ctypes.c_void_p(ptr) if ptr else None)

    def clear(self) -> int:
        return self.lib.sipFftBatchClear(self.b)

    def set_gate(self, flag_ptr: int | None, poll_limit: int = 0) -> int:
        return self.lib.sipFftBatchSetGate(self.b, ctypes.c_void_p(flag_ptr) if flag_ptr else None, poll_limit)

    def take_status(self) -> int:
        s = ctypes.c_uint(0)
        check(self.lib.sipFftBatchTakeStatus(self.b, ctypes.byref(s)), "sipFftBatchTakeStatus")
        return s.value

    def destroy(self) -> None:
        if self.b is not None:
            self.lib.sipFftBatchDestroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

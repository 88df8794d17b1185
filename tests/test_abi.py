"""C ABI without a GPU: the library loads, exports every function its
headers declare, validates like the reference (core/fft/fft_api.cpp) and
builds the expected kernel steps.  Execution on a host without a CUDA
device fails loudly (INTERNAL_ERROR): there is no CPU fallback."""
import ctypes
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

from sip_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]
OK, INV, NOTSUP, INTERNAL = L.ACL_SUCCESS, L.ACL_ERROR_INVALID_PARAM, L.ACL_ERROR_API_NOT_SUPPORT, L.ACL_ERROR_INTERNAL_ERROR
C2C, C2R, R2C, SEP, STFT = L.ASCEND_FFT_C2C, L.ASCEND_FFT_C2R, L.ASCEND_FFT_R2C, L.ASCEND_FFT_C2C_SEP, L.ASCEND_STFT_C2C
F, I = L.ASCEND_FFT_FORWARD, L.ASCEND_FFT_INVERSE


def declared_functions():
    names = set()
    for h in (ROOT / "include").rglob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b((?:asd|acl|sip)[A-Za-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_exports_every_declared_function(sip_lib):
    declared = declared_functions()
    assert {"asdFftCreate", "asdFftExecR2C", "aclCreateTensor", "sipFftExecRaw"} <= declared
    missing = [n for n in declared if not hasattr(sip_lib, n)]
    assert not missing, missing
    assert declared <= set(L.EXPORTED), declared - set(L.EXPORTED)  # the binding covers every entry point
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.LIB_PATH)], capture_output=True, text=True).stdout
    for n in declared:
        assert re.search(rf"\bT {n}$", out, re.M), f"{n} is not an unmangled export"


def test_version(sip_lib):
    assert sip_lib.sipFftVersion().startswith(b"sip_b200-fft")


@pytest.fixture()
def handle(sip_lib):
    h = ctypes.c_void_p()
    assert sip_lib.asdFftCreate(ctypes.byref(h)) == OK
    yield h
    sip_lib.asdFftDestroy(h)


def plan1d(lib, h, n, t=C2C, d=F, b=1, dim=L.ASCEND_FFT_HORIZONTAL):
    return lib.asdFftMakePlan1D(h, n, t, d, b, dim)


def describe(lib, h):
    need = ctypes.c_size_t(0)
    lib.sipFftDescribePlan(h, None, 0, ctypes.byref(need))
    buf = ctypes.create_string_buffer(need.value)
    assert lib.sipFftDescribePlan(h, buf, need.value, ctypes.byref(need)) == OK
    return json.loads(buf.value.decode())


def test_handle_lifecycle(sip_lib):
    h = ctypes.c_void_p()
    assert sip_lib.asdFftCreate(ctypes.byref(h)) == OK and h.value
    assert sip_lib.asdFftDestroy(h) == OK
    assert sip_lib.asdFftDestroy(h) == INV            # already destroyed
    bogus = ctypes.c_void_p(0x1234)
    assert sip_lib.asdFftSetStream(bogus, ctypes.c_void_p(1)) == INV
    assert plan1d(sip_lib, bogus, 64) == INV
    t = ctypes.c_int(0)
    assert sip_lib.asdFftGetType(bogus, ctypes.byref(t)) == INTERNAL
    assert sip_lib.asdFftSynchronize(bogus) == INTERNAL
    sz = ctypes.c_size_t(0)
    assert sip_lib.asdFftGetWorkspaceSize(bogus, ctypes.byref(sz)) == INV
    assert sip_lib.asdFftSetWorkspace(bogus, None) == INV


def test_set_stream_rejects_null(sip_lib, handle):
    assert sip_lib.asdFftSetStream(handle, None) == INV
    assert sip_lib.asdFftSetStream(handle, ctypes.c_void_p(0xdead)) == OK


@pytest.mark.parametrize("n,t,d,b,dim,code", [
    (0, C2C, F, 1, L.ASCEND_FFT_HORIZONTAL, INV),
    ((1 << 27) + 1, C2C, F, 1, L.ASCEND_FFT_HORIZONTAL, INV),
    (64, C2C, F, 0, L.ASCEND_FFT_HORIZONTAL, INV),
    (64, C2C, F, (1 << 31), L.ASCEND_FFT_HORIZONTAL, INV),      # batch above INT32_MAX
    (64, STFT, F, 1, L.ASCEND_FFT_HORIZONTAL, INV),              # STFT types are not 1D FFT types
    (64, 0x99, F, 1, L.ASCEND_FFT_HORIZONTAL, INV),
    (64, C2C, 0x42, 1, L.ASCEND_FFT_HORIZONTAL, INV),            # invalid direction
    (64, C2C, F, 1, 0x42, INV),                                  # invalid dim type
    (64, C2C, F, 4, L.ASCEND_FFT_VERTICAL, NOTSUP),              # vertical batches (Ascend 950 contract)
    (64, C2C, F, 1, L.ASCEND_FFT_VERTICAL, OK),
    (64, C2C, F, 1, L.ASCEND_FFT_HORIZONTAL, OK),
])
def test_make_plan_1d_validation(sip_lib, handle, n, t, d, b, dim, code):
    assert plan1d(sip_lib, handle, n, t, d, b, dim) == code


def test_plan_once(sip_lib, handle):
    assert plan1d(sip_lib, handle, 64) == OK
    assert plan1d(sip_lib, handle, 64) == INV
    assert sip_lib.asdFftMakePlan2D(handle, 8, 8, C2C, F, 1) == INV
    t = ctypes.c_int(0)
    assert sip_lib.asdFftGetType(handle, ctypes.byref(t)) == OK and t.value == C2C


@pytest.mark.parametrize("t,code", [(C2C, OK), (R2C, OK), (C2R, OK), (SEP, INV), (STFT, INV)])
def test_make_plan_2d_types(sip_lib, handle, t, code):
    assert sip_lib.asdFftMakePlan2D(handle, 64, 64, t, F, 1) == code


@pytest.mark.parametrize("args,code", [((0, 8, 8), INV), ((8, 8, 8), OK), ((8, -1, 8), INV)])
def test_make_plan_3d_sizes(sip_lib, handle, args, code):
    assert sip_lib.asdFftMakePlan3D(handle, *args, C2C, F, 1) == code


def test_make_plan_3d_rejects_stft(sip_lib, handle):
    assert sip_lib.asdFftMakePlan3D(handle, 8, 8, 8, STFT, F, 1) == INV


def test_istft_not_supported(sip_lib, handle):
    assert sip_lib.asdFftIstftMakePlan(handle, None, 16, 4, 16, True, False, False, 0, True) == NOTSUP


# ---------------------------------------------------------- tensor checks
class Tensor:
    def __init__(self, lib, shape, dtype, ptr=0x10000):
        n = len(shape)
        dims = (ctypes.c_int64 * max(n, 1))(*shape)
        self.h = lib.aclCreateTensor(dims, n, dtype, None, 0, L.ACL_FORMAT_ND, dims, n, ctypes.c_void_p(ptr))
        self.lib = lib

    def __del__(self):
        self.lib.aclDestroyTensor(self.h)


def test_acl_tensor_shim(sip_lib):
    t = Tensor(sip_lib, [3, 5, 7], L.ACL_COMPLEX64, ptr=0x1000)
    dims = ctypes.POINTER(ctypes.c_int64)()
    n = ctypes.c_uint64(0)
    assert sip_lib.aclGetViewShape(t.h, ctypes.byref(dims), ctypes.byref(n)) == 0
    assert n.value == 3 and [dims[i] for i in range(3)] == [3, 5, 7]
    sip_lib.aclFreeViewShape(dims)
    dt = ctypes.c_int(-1)
    assert sip_lib.aclGetDataType(t.h, ctypes.byref(dt)) == 0 and dt.value == L.ACL_COMPLEX64
    bad = (ctypes.c_int64 * 1)(-2)
    assert not sip_lib.aclCreateTensor(bad, 1, L.ACL_FLOAT, None, 0, L.ACL_FORMAT_ND, bad, 1, None)


def test_exec_tensor_contract(sip_lib, handle):
    """Cross-variant exec, dtype / rank / shape mismatches (reference
    test_fft_c2c_1d.cpp negative cases) are rejected before any device work."""
    assert plan1d(sip_lib, handle, 64, C2C, F, 4) == OK
    ok_in = Tensor(sip_lib, [4, 64], L.ACL_COMPLEX64, 0x10000)
    ok_out = Tensor(sip_lib, [4, 64], L.ACL_COMPLEX64, 0x90000)
    assert sip_lib.asdFftExecR2C(handle, ok_in.h, ok_out.h) == INV              # plan type mismatch
    assert sip_lib.asdFftExecC2R(handle, ok_in.h, ok_out.h) == INV
    for shape, dt in [([4, 64], L.ACL_FLOAT), ([4, 32], L.ACL_COMPLEX64), ([2, 2, 64], L.ACL_COMPLEX64),
                      ([256], L.ACL_COMPLEX64), ([3, 64], L.ACL_COMPLEX64), ([64, 4], L.ACL_COMPLEX64)]:
        bad = Tensor(sip_lib, shape, dt, 0x10000)
        assert sip_lib.asdFftExecC2C(handle, bad.h, ok_out.h) == INV, shape
        assert sip_lib.asdFftExecC2C(handle, ok_in.h, bad.h) == INV, shape
    # valid tensors on a host without a GPU: no CPU fallback
    assert sip_lib.asdFftExecC2C(handle, ok_in.h, ok_out.h) == INTERNAL


def test_batch_one_accepts_both_orientations(sip_lib, handle):
    assert plan1d(sip_lib, handle, 64, C2C, F, 1) == OK
    a = Tensor(sip_lib, [64, 1], L.ACL_COMPLEX64, 0x10000)
    b = Tensor(sip_lib, [1, 64], L.ACL_COMPLEX64, 0x90000)
    assert sip_lib.asdFftExecC2C(handle, a.h, b.h) == INTERNAL   # passes matching, no device


def test_zero_dim_rejected(sip_lib, handle):
    """reference fftzerodim/test_fft_zerodim_negative.cpp:114-137"""
    assert plan1d(sip_lib, handle, 16, C2R, F, 1) == OK
    scalar = Tensor(sip_lib, [], L.ACL_COMPLEX64)
    out = Tensor(sip_lib, [8], L.ACL_FLOAT, 0x90000)
    assert sip_lib.asdFftExecC2R(handle, scalar.h, out.h) == INV


def test_real_tensor_shapes(sip_lib, handle):
    assert plan1d(sip_lib, handle, 30, R2C, F, 6) == OK
    x = Tensor(sip_lib, [2, 3, 30], L.ACL_FLOAT, 0x10000)      # leading dims multiply to the batch
    y = Tensor(sip_lib, [6, 16], L.ACL_COMPLEX64, 0x90000)
    assert sip_lib.asdFftExecR2C(handle, x.h, y.h) == INTERNAL
    y_bad = Tensor(sip_lib, [6, 15], L.ACL_COMPLEX64, 0x90000)
    assert sip_lib.asdFftExecR2C(handle, x.h, y_bad.h) == INV
    x_bad = Tensor(sip_lib, [5, 30], L.ACL_FLOAT, 0x10000)     # batch mismatch
    assert sip_lib.asdFftExecR2C(handle, x_bad.h, y.h) == INV


def test_workspace_protocol(sip_lib, handle):
    """reference fftworkspace/test_fft_workspace_negative.cpp: exec without
    GetWorkspaceSize on a plan that needs scratch is INVALID_PARAM; with the
    size queried but no buffer bound, INTERNAL_ERROR."""
    assert plan1d(sip_lib, handle, 65536, C2C, F, 2) == OK
    x = Tensor(sip_lib, [2, 65536], L.ACL_COMPLEX64, 0x100000)
    y = Tensor(sip_lib, [2, 65536], L.ACL_COMPLEX64, 0x900000)
    assert sip_lib.asdFftExecC2C(handle, x.h, y.h) == INTERNAL     # not bound
    assert sip_lib.asdFftSetWorkspace(handle, ctypes.c_void_p(0x4000000)) == OK
    assert sip_lib.asdFftExecC2C(handle, x.h, y.h) == INV          # size never queried
    sz = ctypes.c_size_t(0)
    assert sip_lib.asdFftGetWorkspaceSize(handle, ctypes.byref(sz)) == OK
    assert sz.value == 2 * 65536 * 8


def test_no_workspace_for_single_pass(sip_lib, handle):
    assert sip_lib.asdFftMakePlan2D(handle, 256, 256, C2C, F, 2) == OK
    sz = ctypes.c_size_t(7)
    assert sip_lib.asdFftGetWorkspaceSize(handle, ctypes.byref(sz)) == OK and sz.value == 0


def test_partial_overlap_rejected(sip_lib, handle):
    assert plan1d(sip_lib, handle, 64, C2C, F, 4) == OK
    x = Tensor(sip_lib, [4, 64], L.ACL_COMPLEX64, 0x10000)
    y = Tensor(sip_lib, [4, 64], L.ACL_COMPLEX64, 0x10000 + 8 * 64)
    assert sip_lib.asdFftExecC2C(handle, x.h, y.h) == INV


@pytest.mark.parametrize("t,sizes,kinds", [
    (C2C, [4096], ["c2c rows"]),
    (C2C, [6000], ["c2c rows"]),
    (C2C, [65536], ["four-step A", "four-step B"]),
    (C2C, [2048, 2048], ["c2c axis 1", "c2c axis 0"]),
    (C2C, [256, 256, 256], ["c2c axis 2", "c2c axis 1", "c2c axis 0"]),
    (R2C, [1000], ["r2c half"]),
    (R2C, [2187], ["r2c pair"]),
    (R2C, [1 << 20], ["four-step A", "r2c four-step B + post"]),
    (C2R, [1 << 20], ["c2r pre", "four-step A", "four-step B"]),
    (C2R, [64, 64], ["c2c axis 0", "c2r half"]),
    # Bluestein up to the largest length (2^27): a convolution of 2^28 in
    # the four-step pulse chain
    (C2C, [(1 << 27) - 1], ["bluestein pre", "four-step A", "pulse rows", "pulse inverse columns",
                            "bluestein post"]),
])
def test_plan_steps(sip_lib, handle, t, sizes, kinds):
    """Every axis is one pass (no transposes); four-step above one tile."""
    if len(sizes) == 1:
        assert plan1d(sip_lib, handle, sizes[0], t, F, 2) == OK
    elif len(sizes) == 2:
        assert sip_lib.asdFftMakePlan2D(handle, *sizes, t, F, 2) == OK
    else:
        assert sip_lib.asdFftMakePlan3D(handle, *sizes, t, F, 1) == OK
    steps = describe(sip_lib, handle)["steps"]
    assert [s["what"].split(" n=")[0] for s in steps] == kinds


def test_compute_mode(sip_lib, handle):
    assert sip_lib.sipFftSetComputeMode(handle, 7) == INV
    assert sip_lib.sipFftSetComputeMode(handle, L.SIP_FFT_COMPUTE_TC_SPLIT) == OK
    assert plan1d(sip_lib, handle, 65536, C2C, F, 2) == OK
    assert all("tensor-core" in s["what"] for s in describe(sip_lib, handle)["steps"])
    assert sip_lib.sipFftSetComputeMode(handle, 0) == INV       # already planned


def test_plan_trace_env():
    code = ("import ctypes,sys; sys.path.insert(0, %r); from sip_b200 import _lib as L; l=L.lib(); "
            "h=ctypes.c_void_p(); l.asdFftCreate(ctypes.byref(h)); l.asdFftMakePlan1D(h, 4096, 0x10, 0x10, 1024, 0x10)"
            % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env={**os.environ, "ASDSIP_FFT_PLAN_TRACE": "1"})
    assert "ASDSIP_FFT_PLAN" in r.stderr and "c2c rows" in r.stderr


def test_plan_hints(sip_lib, handle):
    H = L
    assert sip_lib.sipFftSetPlanHint(handle, 99, 1) == INV
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_ELEMS_PER_THREAD, 8) == INV
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_GENERIC_ONLY, 2) == INV
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_GENERIC_ONLY, 1) == OK
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_ELEMS_PER_THREAD, 32) == OK
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_RADIX_ORDER, 1) == OK
    assert plan1d(sip_lib, handle, 1000, C2C, F, 8) == OK
    (st,) = describe(sip_lib, handle)["steps"]
    assert st["sk"] is False and st["e"] == 32 and st["radices"] == sorted(st["radices"])
    assert sip_lib.sipFftSetPlanHint(handle, H.SIP_FFT_HINT_GENERIC_ONLY, 0) == INV  # already planned


def test_generic_hint_large_real_uses_queueable_passes(sip_lib, handle):
    assert sip_lib.sipFftSetPlanHint(handle, L.SIP_FFT_HINT_GENERIC_ONLY, 1) == OK
    assert plan1d(sip_lib, handle, 1 << 20, R2C, F, 1) == OK
    steps = describe(sip_lib, handle)["steps"]
    assert all(s["sk"] is False for s in steps if s["kind"] == 0)


def test_tune_cache_env(tmp_path):
    cache = tmp_path / "tune.txt"
    cache.write_text("# type dir dims batch P E generic order\n16 16 4096 1024 1 32 1 0\n")
    code = ("import ctypes,sys,json; sys.path.insert(0, %r); from sip_b200.fft import FftHandle; "
            "h=FftHandle(); h.make_plan_1d(4096, 0x10, 0x10, 1024); s=h.describe()['steps'][0]; "
            "print(json.dumps([s['sk'], s['e'], s['P']]))" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env={**os.environ, "SIP_FFT_TUNE_CACHE": str(cache)})
    assert json.loads(r.stdout.strip().splitlines()[-1]) == [False, 32, 1], r.stderr
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=dict(os.environ))
    assert json.loads(r.stdout.strip().splitlines()[-1])[0] is True


def test_tune_cache_runtime_compile_field(tmp_path):
    """The eleventh field of a tune-cache line is the run-time compile hint."""
    cache = tmp_path / "tune.txt"
    cache.write_text("16 16 3840 8192 0 0 0 0 0 0 2\n")
    code = ("import sys,json; sys.path.insert(0, %r); from sip_b200.fft import FftHandle; "
            "h=FftHandle(); h.make_plan_1d(3840, 0x10, 0x10, 8192); s=h.describe()['steps'][0]; "
            "print(json.dumps(s['jit']))" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       env={**os.environ, "SIP_FFT_TUNE_CACHE": str(cache)})
    assert json.loads(r.stdout.strip().splitlines()[-1]) is False, r.stderr


def test_batch_api_without_device(sip_lib, handle):
    b = ctypes.c_void_p()
    assert sip_lib.sipFftBatchCreate(None) == INV
    assert sip_lib.sipFftBatchCreate(ctypes.byref(b)) == INTERNAL  # no CUDA device: no fallback
    assert sip_lib.sipFftBatchExec(None, None) == INV
    assert sip_lib.sipFftBatchAdd(None, handle, None, None) == INV
    assert sip_lib.sipFftBatchTakeStatus(None, None) == INV
    assert sip_lib.sipFftBatchSetGate(None, None, 0) == INV


@pytest.mark.parametrize("t,value,kinds", [
    (C2R, 1, ["c2r pre + four-step A", "four-step B"]),
    (C2R, 2, ["c2r pre", "four-step A", "four-step B"]),
    (R2C, 0, ["four-step A", "r2c four-step B + post"]),
    (R2C, 2, ["four-step A", "four-step B", "r2c post"]),
])
def test_real_fused_hint(sip_lib, handle, t, value, kinds):
    assert sip_lib.sipFftSetPlanHint(handle, L.SIP_FFT_HINT_REAL_FUSED, value) == OK
    assert plan1d(sip_lib, handle, 1 << 20, t, F, 2) == OK
    assert [s["what"].split(" n=")[0] for s in describe(sip_lib, handle)["steps"]] == kinds


def test_bluestein_limit(sip_lib, handle):
    """Lengths above 2^27 are outside the API (the reference's limit); below
    it every length plans, Bluestein's included."""
    assert plan1d(sip_lib, handle, (1 << 27) + 1, C2C, F, 1) == INV
    desc_ok = plan1d(sip_lib, handle, (1 << 27) - 1, C2C, F, 1)
    assert desc_ok == OK
    steps = describe(sip_lib, handle)["steps"]
    assert steps[0]["m"] == 1 << 28


def test_rows_exec_checks(sip_lib, handle):
    """sipFftExecRawRows: rows outside [1, batch] and unplanned handles are
    INVALID_PARAM; plans whose steps cannot be limited to rows (multi-D,
    Bluestein lengths) are API_NOT_SUPPORT; all before touching a device."""
    x, y = ctypes.c_void_p(0x10000), ctypes.c_void_p(0x40000000)
    assert sip_lib.sipFftExecRawRows(handle, 1, x, y, None) == INV   # not planned
    assert plan1d(sip_lib, handle, 4096, C2C, F, 8) == OK
    for rows in (0, -1, 9):
        assert sip_lib.sipFftExecRawRows(handle, rows, x, y, None) == INV
    h2 = ctypes.c_void_p()
    assert sip_lib.asdFftCreate(ctypes.byref(h2)) == OK
    assert sip_lib.asdFftMakePlan2D(h2, 64, 64, C2C, F, 2) == OK
    assert sip_lib.sipFftExecRawRows(h2, 1, x, y, None) == NOTSUP
    sip_lib.asdFftDestroy(h2)
    h3 = ctypes.c_void_p()
    assert sip_lib.asdFftCreate(ctypes.byref(h3)) == OK
    assert plan1d(sip_lib, h3, 100003, C2C, F, 2) == OK   # prime: Bluestein steps
    assert sip_lib.sipFftExecRawRows(h3, 1, x, y, None) == NOTSUP
    sip_lib.asdFftDestroy(h3)


@pytest.mark.parametrize("t,n", [(R2C, 1 << 20), (C2R, 1 << 20), (C2C, 65536), (R2C, 6000), (C2R, 1000),
                                 (C2C, 4096)])
def test_rows_exec_supported_for_1d_plans(sip_lib, handle, t, n):
    """Every 1-D plan of a benchmark length can run on its first rows: the
    row-limited exec passes its plan checks and stops only at the missing
    device (or workspace), not with API_NOT_SUPPORT."""
    assert plan1d(sip_lib, handle, n, t, F if t != C2R else L.ASCEND_FFT_INVERSE, 4) == OK
    rc = sip_lib.sipFftExecRawRows(handle, 2, ctypes.c_void_p(0x10000), ctypes.c_void_p(0x40000000), None)
    assert rc == INTERNAL, rc

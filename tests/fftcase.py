"""Shared helpers of the tests: run one transform through the C ABI on the
GPU, or through the CPU harness, and compare with the oracle."""
from __future__ import annotations

import ctypes
import json

import numpy as np

from oracle import oracle as O
from sip_b200 import _lib as L

TYPES = {"c2c": O.C2C, "r2c": O.R2C, "c2r": O.C2R}
DIRS = {"fwd": O.FORWARD, "inv": O.INVERSE}


def shapes(op: int, sizes, batch: int):
    """(input shape, input dtype, output shape, output dtype) as the reference's tensors."""
    lead = (batch,)
    full = lead + tuple(sizes)
    half = lead + tuple(sizes[:-1]) + (sizes[-1] // 2 + 1,)
    if op == O.C2C:
        return full, np.complex64, full, np.complex64
    if op == O.R2C:
        return full, np.float32, half, np.complex64
    return half, np.complex64, full, np.float32


def random_input(op: int, sizes, batch: int, seed: int = 20261029):
    rng = np.random.default_rng(seed)
    ishape, idt, _, _ = shapes(op, sizes, batch)
    if idt == np.float32:
        return rng.uniform(-1, 1, ishape).astype(np.float32)
    return (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64)


def emu_run(emu, op: int, direction: int, sizes, batch: int, x: np.ndarray):
    _, _, oshape, odt = shapes(op, sizes, batch)
    out = np.zeros(oshape, odt)
    sz = (ctypes.c_longlong * len(sizes))(*sizes)
    desc = ctypes.create_string_buffer(1 << 16)
    xc = np.ascontiguousarray(x)
    rc = emu.emu_exec(op, direction, len(sizes), sz, batch, xc.ctypes.data, out.ctypes.data, desc, len(desc))
    return rc, out, desc.value.decode()


def make_plan(h, op: int, direction: int, sizes, batch: int) -> int:
    if len(sizes) == 1:
        return h.make_plan_1d(sizes[0], op, direction, batch)
    if len(sizes) == 2:
        return h.make_plan_2d(sizes[0], sizes[1], op, direction, batch)
    return h.make_plan_3d(sizes[0], sizes[1], sizes[2], op, direction, batch)


def settle() -> None:
    """Waits for all work on the device.  The library runs on its own
    (non-default) stream, so inputs and outputs that torch filled on the
    default stream must be complete before a test launches on it."""
    import torch

    torch.cuda.synchronize()


def gpu_run(torch, op: int, direction: int, sizes, batch: int, x: np.ndarray, stream=None, keep=False):
    """Plan -> workspace -> stream -> exec through aclTensors -> sync -> destroy."""
    from sip_b200.fft import FftHandle, check

    _, _, oshape, odt = shapes(op, sizes, batch)
    dev = torch.device("cuda")
    xt = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    yt = torch.zeros(oshape, dtype=torch.complex64 if odt == np.complex64 else torch.float32, device=dev)
    h = FftHandle()
    check(make_plan(h, op, direction, list(sizes), batch), "make plan")
    h.bind_workspace()
    s = stream or torch.cuda.Stream()
    check(h.set_stream(s), "set stream")
    fn = {O.C2C: h.exec_c2c, O.R2C: h.exec_r2c, O.C2R: h.exec_c2r}[op]
    settle()
    check(fn(xt, yt), "exec")
    check(h.synchronize(), "synchronize")
    out = yt.cpu().numpy()
    if keep:
        return out, h, xt, yt
    h.destroy()
    return out

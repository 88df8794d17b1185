"""L2-resident chunks of multi-step plans, on the CPU harness.

Steps of a chunk group (the passes of a four-step transform, of a pulse
chain, of a large real transform with its pre/post pass, the axis passes of
a 2-D / 3-D transform) run chunk by chunk, each chunk on a slice of the
batch rows, items or slabs, reusing one workspace region.  The harness runs
the library's planner and the same chunk order as the library's launcher,
with the workspace filled with NaN: a chunk that read anything no step of
it wrote would show up.  Every result must match the FP64 oracle and the
unchunked run bit for bit.
"""
import ctypes
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests.fftcase import emu_run, random_input

REL_L2_TOL = 1e-6

CASES = [  # (type, direction, sizes, batch, chunk bytes)
    (O.C2C, O.FORWARD, [32768], 5, 2 * 32768 * 8),
    (O.C2C, O.INVERSE, [65536], 3, 65536 * 8),
    (O.R2C, O.FORWARD, [65536], 3, 32768 * 8),
    (O.C2R, O.INVERSE, [65536], 3, 32768 * 8),
    (O.C2R, O.FORWARD, [65536], 5, 2 * 32768 * 8),
    (O.C2C, O.FORWARD, [64, 48], 5, 2 * 64 * 48 * 8),
    (O.C2C, O.INVERSE, [40, 36], 4, 40 * 36 * 8),
    (O.R2C, O.FORWARD, [64, 48], 5, 2 * 64 * 48 * 8),
    (O.C2R, O.INVERSE, [64, 48], 5, 2 * 64 * 48 * 8),
    (O.C2C, O.FORWARD, [16, 12, 20], 1, 4 * 12 * 20 * 8),  # slabs of the outermost axis
    (O.R2C, O.FORWARD, [16, 12, 20], 2, 3 * 12 * 11 * 8),
    (O.C2C, O.FORWARD, [16, 12, 20], 3, 16 * 12 * 20 * 8),  # whole items
]


def run(emu, typ, d, sizes, batch, x, chunk):
    emu.emu_set_chunk_bytes(chunk)
    try:
        return emu_run(emu, typ, d, sizes, batch, x)
    finally:
        emu.emu_set_chunk_bytes(-1)


@pytest.mark.parametrize("typ,d,sizes,batch,chunk", CASES)
def test_chunked_plans_match_oracle_and_unchunked(emu, typ, d, sizes, batch, chunk):
    x = random_input(typ, sizes, batch, seed=sum(sizes) + batch)
    rc, out, desc = run(emu, typ, d, sizes, batch, x, chunk)
    assert rc == 0, desc
    plan = json.loads(desc)
    assert plan["chunk_groups"], desc[:600]
    assert plan["launches"] > len(plan["steps"]), desc[:600]  # more than one chunk
    assert O.rel_l2(out, O.fp64(typ, d, x, sizes)) <= REL_L2_TOL
    rc0, out0, desc0 = run(emu, typ, d, sizes, batch, x, 0)  # chunking off
    assert rc0 == 0 and json.loads(desc0)["launches"] == len(json.loads(desc0)["steps"])
    assert np.array_equal(out, out0)


def test_pulse_chain_chunked(emu):
    n, batch = 32768, 3
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((batch, n)) + 1j * rng.standard_normal((batch, n))).astype(np.complex64)
    filt = O.chirp_spectrum(n).astype(np.complex64)
    out = np.zeros_like(x)
    desc = ctypes.create_string_buffer(1 << 16)
    emu.emu_exec_pulse.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    emu.emu_set_chunk_bytes(n * 8)
    try:
        rc = emu.emu_exec_pulse(n, batch, filt.ctypes.data, 1, x.ctypes.data, out.ctypes.data, desc, len(desc))
    finally:
        emu.emu_set_chunk_bytes(-1)
    assert rc == 0
    plan = json.loads(desc.value.decode())
    assert plan["launches"] == 3 * batch
    assert O.rel_l2(out, O.pulse(x, filt, conj=True)) <= REL_L2_TOL

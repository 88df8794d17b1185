"""CPU tests of the kernel arithmetic: the library's planner and the
kernels' own host-device phase functions, driven on the CPU by
tests/native/tile_emu.cpp, against the oracle.

Covers every reference unit-test case plus plan kinds the GPU suite runs
at full size only (four-step, large real, multi-D real, odd batches)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tests import ref_cases as RC
from tests.fftcase import emu_run, random_input, shapes

REL_L2_TOL = 1e-6


def _check(emu, op, direction, sizes, batch, x=None):
    if x is None:
        ishape, idt, _, _ = shapes(op, sizes, batch)
        x = O.ut_input(ishape, idt)
    rc, out, desc = emu_run(emu, op, direction, sizes, batch, x)
    assert rc == 0, desc
    gold = O.golden(op, direction, x, sizes)
    err = O.rel_l2(out, O.fp64(op, direction, x, sizes))
    assert O.ref_check_mismatches(out, gold) == 0, f"rel_l2={err:.3e} {desc[:300]}"
    assert err <= REL_L2_TOL, desc[:300]


@pytest.mark.parametrize("batch,n,direction", RC.C2C_1D)
def test_ref_c2c_1d(emu, batch, n, direction):
    _check(emu, O.C2C, direction, [n], batch)


@pytest.mark.parametrize("batch,n,direction", RC.R2C_1D)
def test_ref_r2c_1d(emu, batch, n, direction):
    _check(emu, O.R2C, direction, [n], batch)


@pytest.mark.parametrize("batch,n,direction", RC.C2R_1D)
def test_ref_c2r_1d(emu, batch, n, direction):
    _check(emu, O.C2R, direction, [n], batch)


@pytest.mark.parametrize("x,y,batch,direction", RC.C2C_2D)
def test_ref_c2c_2d(emu, x, y, batch, direction):
    _check(emu, O.C2C, direction, [x, y], batch)


@pytest.mark.parametrize("x,y,z,batch,direction", RC.C2C_3D)
def test_ref_c2c_3d(emu, x, y, z, batch, direction):
    _check(emu, O.C2C, direction, [x, y, z], batch)


@pytest.mark.parametrize("op", [O.C2C, O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
@pytest.mark.parametrize("sizes,batch", [([1], 3), ([2], 5), ([3], 4), ([7], 3), ([1000], 5), ([2187], 3),
                                         ([6000], 2), ([65536], 1), ([40000], 1), ([8, 8], 3), ([30, 33], 3),
                                         ([9, 7, 5], 2), ([1, 12], 2), ([5, 1, 4], 1),
                                         ([2944], 2), ([2976], 2), ([1856], 2), ([667], 3), ([961], 2)])
def test_plan_kinds(emu, op, direction, sizes, batch):
    x = random_input(op, sizes, batch, seed=sum(sizes) + batch)
    _check(emu, op, direction, sizes, batch, x)


def test_radix_butterflies(emu):
    rng = np.random.default_rng(3)
    from sip_b200.build import CSRC

    text = (CSRC / "fft_core.cuh").read_text()
    line = [l for l in text.splitlines() if l.strip().startswith("X(2)")][0]
    radices = [int(t.strip("X()")) for t in line.split()]
    assert radices
    for r in radices:
        for sign in (-1, 1):
            x = (rng.standard_normal(r) + 1j * rng.standard_normal(r)).astype(np.complex64)
            y = x.copy()
            assert emu.emu_dft(r, sign, y.ctypes.data) == 0
            ref = np.fft.fft(x.astype(np.complex128)) if sign < 0 else np.fft.ifft(x.astype(np.complex128)) * r
            assert O.rel_l2(y, ref) < 2e-7, r


def test_fastdiv_exact(emu):
    rng = np.random.default_rng(5)
    d = np.concatenate([np.arange(1, 5000, dtype=np.uint32), rng.integers(1, 2**31 - 1, 20000).astype(np.uint32)])
    n = np.concatenate([rng.integers(0, 2**32 - 1, d.size).astype(np.uint32)])
    edge_d = np.repeat(np.array([1, 2, 3, 7, 641, 65537, 2**31 - 1], np.uint32), 6)
    edge_n = np.tile(np.array([0, 1, 2**31 - 1, 2**31, 2**32 - 2, 2**32 - 1], np.uint32), 7)
    d = np.ascontiguousarray(np.concatenate([d, edge_d]))
    n = np.ascontiguousarray(np.concatenate([n, edge_n]))
    assert emu.emu_fastdiv_check(d.ctypes.data, n.ctypes.data, d.size) == 0


def _sk_list(emu):
    import ctypes

    emu.emu_sk_list.argtypes = [ctypes.c_void_p, ctypes.c_int]
    buf = np.zeros(7 * 256, np.int32)
    n = emu.emu_sk_list(buf.ctypes.data, 256)
    return [tuple(int(v) for v in buf[7 * i:7 * i + 7]) for i in range(n)]


def _plan_for_sk(op, mode, sign, tw4, n):
    """(type, direction, sizes, batch) of a plan whose steps include this kernel."""
    d = O.FORWARD if sign < 0 else O.INVERSE
    if op == 5:  # R2C four-step pass B with the mirrored post-process
        return O.R2C, O.INVERSE, [2 * (1 << 19)], 3
    if op == 6:  # C2R pre-process with the mirrored four-step pass A
        return O.C2R, O.FORWARD, [2 * (1 << 19)], 3
    if mode == 0:  # rows
        if op == 0:
            return O.C2C, d, [n], 37
        if op == 1:
            return O.R2C, O.INVERSE, [2 * n], 21
        if op == 2:
            return O.C2R, O.FORWARD, [2 * n], 21
        if op == 3:
            return O.R2C, O.FORWARD, [n], 9
        return O.C2R, O.INVERSE, [n], 9
    if mode == 1 and not tw4:
        return O.C2C, d, [n, 24], 2
    split = {256: 65536, 512: 1 << 19, 1024: 1 << 19}
    return O.C2C, d, [split[n]], 1


def _split_n1(op, mode, tw4, n):
    """Column length of the four-step split that uses this kernel, when it
    is not the planner's default (2^19 = 512 x 1024)."""
    if n == 512 and ((op == 5 and mode == 2) or (op == 0 and mode == 2)):
        return 1024   # rows of 512
    if n == 1024 and op == 0 and mode == 1 and tw4:
        return 1024   # columns of 1024
    return None


def test_every_specialized_kernel(emu, monkeypatch):
    """Each compiled size-specialized kernel is selected by the planner and
    matches the FP64 oracle (including partial tiles and odd row counts).
    The opt-in cluster form stays off here (tests/test_emu_cluster.py
    covers it)."""
    monkeypatch.delenv("SIP_FFT_CLUSTER", raising=False)
    entries = _sk_list(emu)
    assert len(entries) >= 20
    emu.emu_set_real_fused.argtypes = [ctypes.c_int]
    emu.emu_set_sk_variant.argtypes = [ctypes.c_int]
    seen = {}
    for op, mode, sign, tw4, n, P, T in entries:
        if op == 7:  # pulse-compression tiles: test_emu_pulse.py / test_emu_bluestein.py
            continue
        typ, d, sizes, batch = _plan_for_sk(op, mode, sign, tw4, n)
        x = random_input(typ, sizes, batch, seed=n + op)
        key = (op, mode, sign, tw4, n)
        variant = seen.get(key, 0)  # later entries of the same kernel are hint-selected variants
        seen[key] = variant + 1
        emu.emu_set_real_fused(1 if op == 6 else 0)  # the fused C2R form is selected by hint
        emu.emu_set_sk_variant(variant)
        n1 = _split_n1(op, mode, tw4, n)
        if n1:
            monkeypatch.setenv("SIP_FFT_SPLIT_N1", str(n1))
        else:
            monkeypatch.delenv("SIP_FFT_SPLIT_N1", raising=False)
        try:
            rc, out, desc = emu_run(emu, typ, d, sizes, batch, x)
        finally:
            emu.emu_set_real_fused(0)
            emu.emu_set_sk_variant(-1)
        assert rc == 0, desc
        import json

        steps = json.loads(desc)["steps"]
        hit = [s for s in steps if s.get("sk") and s["n"] == n and s["op"] == op and s["sign"] == sign
               and s["tw4"] == bool(tw4) and s["P"] * (2 if op in (5, 6) else 1) == P and s["threads"] == T]
        assert hit, (op, mode, sign, tw4, n, desc[:400])
        err = O.rel_l2(out, O.fp64(typ, d, x, sizes))
        assert err <= REL_L2_TOL, (op, mode, sign, tw4, n, err)

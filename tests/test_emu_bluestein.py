"""Lengths with a prime factor above 32 run Bluestein's algorithm
(bluestein.cuh): CPU harness against the FP64 oracle, C2C / R2C / C2R,
both directions, single-tile and four-step convolution lengths."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests.fftcase import emu_run, random_input

REL_L2_TOL = 1e-6
# odd lengths run the full-length complex transform for R2C / C2R; even
# ones (2018, 8198, 40022) the half-length one between the real pre / post
# passes
LENGTHS = [37, 67, 97, 629, 1009, 2018, 4099, 8198, 20011, 40022]


@pytest.mark.parametrize("n", LENGTHS)
@pytest.mark.parametrize("op", [O.C2C, O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_bluestein_harness(emu, n, op, direction):
    batch = 3
    x = random_input(op, [n], batch, seed=n + op)
    if op == O.C2R:  # a genuine half spectrum (imaginary DC / Nyquist ignored as numpy does)
        x = np.fft.rfft(np.random.default_rng(n).uniform(-1, 1, (batch, n))).astype(np.complex64)
    rc, out, desc = emu_run(emu, op, direction, [n], batch, x)
    assert rc == 0, desc
    kinds = [s["what"].split(" n=")[0] for s in json.loads(desc)["steps"]]
    # fused: one size-specialized pulse tile with the chirps on load and
    # store (the harness instantiates the tile of m = 2025, n = 1009);
    # otherwise pre pass, convolution, post pass
    fused = "bluestein" in kinds
    assert fused or ("bluestein pre" in kinds and "bluestein post" in kinds), kinds
    assert fused == ((op == O.C2C and n == 1009) or (op != O.C2C and n == 2018)), kinds
    if op != O.C2C and n % 2 == 0:  # half length between the real passes
        blue = "bluestein" if fused else "bluestein pre"
        assert kinds[0] == ("c2r pre" if op == O.C2R else blue), kinds
        assert kinds[-1] == (("bluestein" if fused else "bluestein post") if op == O.C2R else "r2c post"), kinds
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, err


@pytest.mark.parametrize("n", [1000, 2944, 2976, 1856])  # 2^7 23, 2^5 3 31, 2^6 29 have prime radix passes
def test_direct_lengths_do_not_use_bluestein(emu, n):
    x = random_input(O.C2C, [n], 2)
    rc, _, desc = emu_run(emu, O.C2C, O.FORWARD, [n], 2, x)
    assert rc == 0 and "bluestein" not in desc


# Multi-dimensional C2C whose contiguous last axis is above one tile (the
# batched 1-D four-step of the rows) or needs Bluestein, then the column
# passes of the other axes in place on the destination.
@pytest.mark.parametrize("sizes,batch", [([4, 20011], 2), ([3, 5, 1009], 1), ([3, 40000], 2), ([2, 3, 65536], 1)])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_multid_large_or_bluestein_last_axis(emu, sizes, batch, direction):
    x = random_input(O.C2C, sizes, batch, seed=sum(sizes) + batch)
    rc, out, desc = emu_run(emu, O.C2C, direction, sizes, batch, x)
    assert rc == 0, desc
    kinds = [s["what"].split(" n=")[0] for s in json.loads(desc)["steps"]]
    last = sizes[-1]
    if last in (20011, 1009):
        assert any(k.startswith("bluestein") for k in kinds), kinds
    else:
        assert kinds[:2] == ["four-step A", "four-step B"], kinds
    assert kinds[-(len(sizes) - 1):] == [f"c2c axis {ax}" for ax in range(len(sizes) - 2, -1, -1)], kinds
    err = O.rel_l2(out, O.fp64(O.C2C, direction, x, sizes))
    assert err <= REL_L2_TOL, err


# Multi-dimensional real plans whose last axis is above one tile (even: the
# half-length transform; odd, 59049 = 3^10: row pairs through the complex
# four-step) or needs Bluestein (2018 and 40022 at half length, 1009 at
# full length), before (R2C) or after (C2R) the column passes on the half
# spectrum.
@pytest.mark.parametrize("sizes,batch", [([3, 40000], 2), ([2, 3, 65536], 1), ([3, 59049], 1), ([2, 2, 59049], 1),
                                         ([3, 2018], 2), ([2, 3, 1009], 1), ([5, 40022], 1)])
@pytest.mark.parametrize("op", [O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_multid_real_large_last_axis(emu, sizes, batch, op, direction):
    x = random_input(op, sizes, batch, seed=sum(sizes) + batch)
    if op == O.C2R:  # genuine half spectra of real data (imaginary DC / Nyquist as numpy drops them)
        x = np.fft.rfftn(np.random.default_rng(sum(sizes)).uniform(-1, 1, [batch] + sizes),
                         axes=list(range(1, len(sizes) + 1))).astype(np.complex64)
    rc, out, desc = emu_run(emu, op, direction, sizes, batch, x)
    assert rc == 0, desc
    kinds = [s["what"].split(" n=")[0] for s in json.loads(desc)["steps"]]
    cols = [f"c2c axis {ax}" for ax in range(len(sizes) - 2, -1, -1)]
    assert (kinds[-len(cols):] if op == O.R2C else kinds[:len(cols)]) == cols, kinds
    err = O.rel_l2(out, O.fp64(op, direction, x, sizes))
    assert err <= REL_L2_TOL, err

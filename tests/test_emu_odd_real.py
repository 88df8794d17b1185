"""Odd real lengths above one tile on the CPU harness: two real rows as one
complex row through the complex four-step between element-wise passes (R2C
pack / separate, C2R combine / split), both directions, odd and even row
counts (the last pair holding one row)."""
import json

import pytest

from oracle import oracle as O
from tests.fftcase import emu_run, random_input

REL_L2_TOL = 1e-6


@pytest.mark.parametrize("n", [59049, 98415])
@pytest.mark.parametrize("op,direction", [(O.R2C, O.FORWARD), (O.R2C, O.INVERSE), (O.C2R, O.INVERSE),
                                          (O.C2R, O.FORWARD)])
@pytest.mark.parametrize("batch", [1, 2, 3])
def test_odd_real_above_one_tile(emu, n, op, direction, batch):
    x = random_input(op, [n], batch, seed=n + batch)
    rc, out, desc = emu_run(emu, op, direction, [n], batch, x)
    assert rc == 0, desc
    kinds = [s["what"].split(" n=")[0] for s in json.loads(desc)["steps"]]
    first, last = ("r2c pair pack", "r2c pair separate") if op == O.R2C else ("c2r pair combine", "c2r pair split")
    assert kinds == [first, "four-step A", "four-step B", last], kinds
    assert O.rel_l2(out, O.fp64(op, direction, x, [n])) <= REL_L2_TOL

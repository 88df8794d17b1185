"""Randomized plans on the CPU harness: any length 1..6000 (radix passes,
pair/half real paths, Bluestein for large prime factors), any batch, every
type and direction, against the FP64 oracle."""
import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

from oracle import oracle as O
from tests.fftcase import emu_run, random_input

REL_L2_TOL = 1e-6


@settings(max_examples=80, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(n=st.integers(1, 6000), batch=st.integers(1, 5), op=st.sampled_from([O.C2C, O.R2C, O.C2R]),
       direction=st.sampled_from([O.FORWARD, O.INVERSE]))
def test_random_plans(emu, n, batch, op, direction):
    if op == O.C2R:
        x = np.fft.rfft(np.random.default_rng(n).uniform(-1, 1, (batch, n))).astype(np.complex64)
    else:
        x = random_input(op, [n], batch, seed=n * 7 + batch)
    rc, out, desc = emu_run(emu, op, direction, [n], batch, x)
    assert rc == 0, desc
    want = O.fp64(op, direction, x, [n])
    if np.abs(want).max() == 0:
        assert np.abs(out).max() == 0
        return
    assert O.rel_l2(out, want) <= REL_L2_TOL, (n, batch, op, direction)

"""The oracle is pinned before it is trusted (CPU only):
  - its LCG reproduces the reference unit tests' inputs (committed head),
  - numpy goldens of reference unit-test cases match the committed fixtures,
  - its C restatement of the reference's Stockham arithmetic matches the
    outputs of the reference's own Stockham core (compiled on the CPU;
    committed fixtures, regenerated by tests/golden/make_golden.py) and the
    FP64 oracle on the reference's whole case lists,
  - the reference's elementwise check behaves like numpy.isclose."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from tests import ref_cases as RC
from tests.golden import make_golden as MG

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")


def test_lcg_head_pinned():
    assert np.array_equal(O.lcg_uniform(64), GOLD["lcg_head"])
    v = O.lcg_uniform(3)
    # state 2026 * 1664525 + 1013904223 = 4386231873 -> mod 2^32 = 91264577
    assert abs(v[0] - (-300.0 + 91264577 / 2**32 * 600.0)) < 1e-3


@pytest.mark.parametrize("case", MG.CASES, ids=lambda c: MG.case_key(*c))
def test_goldens_pinned(case):
    op, sizes, batch, d = case
    x = MG.case_input(op, sizes, batch)
    code = {"c2c": O.C2C, "r2c": O.R2C, "c2r": O.C2R}[op]
    g = GOLD[MG.case_key(*case) + "__golden"]
    assert O.ref_check_mismatches(O.golden(code, d, x, sizes), g) == 0
    assert O.rel_l2(O.fp64(code, d, x, sizes), g) < 1e-6


@pytest.mark.parametrize("m", MG.REF_M)
@pytest.mark.parametrize("direction", ["fwd", "inv"])
def test_restatement_matches_reference_stockham(m, direction):
    """oracle/stockham.c (FP32, the reference's stage order and tables) vs the
    reference's own Stockham core on the same LCG row."""
    x = O.ut_input((1, m), np.complex64)
    ref = GOLD[f"ref_m{m}_{direction}"]
    mine = O.stockham(O.C2C, O.FORWARD if direction == "fwd" else O.INVERSE, x, m)
    assert O.rel_l2(mine, ref) < 2e-7
    if O.ref_lib() is not None:  # the live reference build, where its sources exist
        live = O.ref_stockham_c2c(x, inverse=direction == "inv")
        assert np.array_equal(live, ref)


@pytest.mark.parametrize("op,cases", [(O.C2C, RC.C2C_1D), (O.R2C, RC.R2C_1D), (O.C2R, RC.C2R_1D)])
def test_restatement_on_reference_cases(op, cases):
    from tests.fftcase import shapes

    for batch, n, d in cases:
        ishape, idt, _, _ = shapes(op, [n], batch)
        x = O.ut_input(ishape, idt)
        ref = O.fp64(op, d, x, [n])
        assert O.rel_l2(O.stockham(op, d, x, n, fp64_math=True), ref) < 1e-12
        out32 = O.stockham(op, d, x, n)
        assert O.rel_l2(out32, ref) < 1e-6
        assert O.ref_check_mismatches(out32, O.golden(op, d, x, [n])) == 0


def test_isclose_semantics():
    g = np.array([1.0, 100.0, 0.0, np.nan], np.float32)
    o = np.array([1.0005, 100.2, 2e-5, np.nan], np.float32)
    # 1.0005 within 1e-5 + 1e-3; 100.2 outside 1e-5 + 0.1; 2e-5 outside 1e-5; NaN never matches
    assert O.isclose_mismatches(o, g) == 3


def test_known_answer_patterns():
    x, g = O.kat_input("impulse", O.C2C, 64, 2)
    assert np.allclose(g, np.exp(-2j * np.pi * np.arange(64) / 64) * (1 + 1j))
    x, g = O.kat_input("constant", O.R2C, 64, 1)
    assert abs(g[0, 0] - 64) < 1e-12 and np.abs(g[0, 1:]).max() < 1e-12

"""Generates the golden fixtures of tests/golden/ (run in a checkout that
has the reference sources, so oracle/_ref is built).

golden.npz holds
  lcg_head            first 64 values of the reference unit tests' LCG
                      (state 2026, U[-300, 300)), float32
  <case>__golden      numpy.fft golden of a reference unit-test case on its
                      LCG input, computed in FP64 and cast like gen_data.py
  ref_m<M>_<dir>      output of the reference's own Stockham core
                      (ops/fft/real/fft_stockham/.../fft_stockham_mix.h, run on
                      the CPU through oracle/_ref) for one LCG row of length M
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

CASES = [
    ("c2c", [64], 1, O.FORWARD), ("c2c", [81], 1, O.INVERSE), ("c2c", [125], 1, O.FORWARD),
    ("c2c", [17], 1, O.INVERSE), ("c2c", [210], 2, O.FORWARD), ("c2c", [360], 1, O.FORWARD),
    ("c2c", [1024], 2, O.INVERSE), ("r2c", [16], 2, O.FORWARD), ("r2c", [27], 4, O.FORWARD),
    ("r2c", [210], 8, O.INVERSE), ("c2r", [16], 2, O.INVERSE), ("c2r", [30], 2, O.FORWARD),
    ("c2r", [27], 1, O.INVERSE), ("c2c", [32, 48], 2, O.FORWARD), ("c2c", [8, 8, 8], 1, O.FORWARD),
]
REF_M = [1500, 2187, 3000]


def case_key(op, sizes, batch, d):
    return f"{op}_{'x'.join(map(str, sizes))}_b{batch}_{'fwd' if d == O.FORWARD else 'inv'}"


def case_input(op, sizes, batch):
    from tests.fftcase import shapes

    ishape, idt, _, _ = shapes({"c2c": O.C2C, "r2c": O.R2C, "c2r": O.C2R}[op], sizes, batch)
    return O.ut_input(ishape, idt)


def main():
    out = {"lcg_head": O.lcg_uniform(64)}
    for op, sizes, batch, d in CASES:
        x = case_input(op, sizes, batch)
        code = {"c2c": O.C2C, "r2c": O.R2C, "c2r": O.C2R}[op]
        g = O.fp64(code, d, x, sizes)
        out[case_key(op, sizes, batch, d) + "__golden"] = g.astype(np.complex64 if code != O.C2R else np.float32)
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref is not built (needs the reference sources): run `make -C oracle`")
    for m in REF_M:
        x = O.ut_input((1, m), np.complex64)
        for d, name in ((False, "fwd"), (True, "inv")):
            out[f"ref_m{m}_{name}"] = O.ref_stockham_c2c(x, inverse=d)
    np.savez_compressed(HERE / "golden.npz", **out)
    print(HERE / "golden.npz", sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()

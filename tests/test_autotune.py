"""Autotuner: candidate set, cache lines the planner reads back (CPU, with a
modelled timer), and a real tuning run on the GPU."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from sip_b200 import _lib as L
from sip_b200.autotune import Candidate, candidates, tune

ROOT = Path(__file__).resolve().parents[1]


def test_candidates_cover_the_hints():
    cs = candidates()
    assert cs[0] == Candidate() and len(set(cs)) == len(cs)
    assert {c.e for c in cs} == {0, 16, 32} and {c.order for c in cs} == {0, 1}
    assert {c.p for c in cs} >= {0, 1, 2, 4, 8, 16}
    assert {c.fused for c in cs} == {0, 1, 2}


def test_fastest_candidate_is_cached_and_read_back(tmp_path):
    cache = tmp_path / "tune.txt"
    want = Candidate(p=2, e=32, generic=1, order=1)
    r = tune(L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, [4096], 64, str(cache),
             timer=lambda c: 1.0 if c == want else 2.0)
    assert r["best"] == want
    assert cache.read_text() == "16 16 4096 64 2 32 1 1 0 -1 0\n"
    code = ("import sys,json; sys.path.insert(0, %r); from sip_b200.fft import FftHandle; h=FftHandle(); "
            "h.make_plan_1d(4096, 0x10, 0x10, 64); s=h.describe()['steps'][0]; "
            "print(json.dumps([s['sk'], s['e'], s['P'], s['radices']]))" % str(ROOT))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         env={**os.environ, "SIP_FFT_TUNE_CACHE": str(cache)}).stdout
    sk, e, p, radices = json.loads(out.strip().splitlines()[-1])
    assert (sk, e, p) == (False, 32, 2) and radices == sorted(radices)


def test_no_candidate_raises():
    with pytest.raises(RuntimeError):
        tune(L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, [64], 1, None, timer=lambda c: float("inf"))


@pytest.mark.gpu
def test_tune_on_gpu(cuda, tmp_path):
    cache = tmp_path / "tune.txt"
    r = tune(L.ASCEND_FFT_R2C, L.ASCEND_FFT_FORWARD, [1000], 4096, str(cache), reps=5)
    assert r["ms"] > 0 and r["ms"] <= r["times"][Candidate()] + 1e-9
    assert cache.read_text().startswith("18 16 1000 4096 ")

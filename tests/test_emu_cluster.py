"""The cluster four-step (one C2C transform per thread-block cluster, the CTAs
exchanging through distributed shared memory) on the CPU harness: the
kernel's phases run rank by rank with the cluster's shared memories as host
buffers.  With SIP_FFT_CLUSTER=1, plans of the compiled lengths pick it;
by default they keep one CTA per transform (measured faster on B200)."""
import json

import pytest

from oracle import oracle as O
from tests.fftcase import emu_run, random_input

REL_L2_TOL = 1e-6


@pytest.mark.parametrize("n,batch", [(1024, 3), (4096, 5), (8192, 2), (4096, 1)])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_cluster_c2c(emu, n, batch, direction, monkeypatch):
    monkeypatch.setenv("SIP_FFT_CLUSTER", "1")
    x = random_input(O.C2C, [n], batch, seed=n + batch)
    rc, out, desc = emu_run(emu, O.C2C, direction, [n], batch, x)
    assert rc == 0, desc
    steps = json.loads(desc)["steps"]
    assert len(steps) == 1 and steps[0]["kind"] == 9, desc[:300]
    assert O.rel_l2(out, O.fp64(O.C2C, direction, x, [n])) <= REL_L2_TOL


def test_cluster_form_is_opt_in(emu, monkeypatch):
    from sip_b200 import _lib as L
    from sip_b200.fft import FftHandle

    monkeypatch.delenv("SIP_FFT_CLUSTER", raising=False)
    for n, batch in ((4096, 2), (4096, 1024)):
        h = FftHandle()
        assert h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, batch) == 0
        assert h.describe()["steps"][0]["kind"] == 0
        h.destroy()
    monkeypatch.setenv("SIP_FFT_CLUSTER", "1")
    h = FftHandle()
    assert h.make_plan_1d(4096, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 1024) == 0
    assert h.describe()["steps"][0]["kind"] == 9
    h.destroy()

"""sipFftExecRawRows: a resident plan run on the first rows of its batch.

The serving loop keeps one plan per length at its largest batch and runs
every request's rows through it.  For each kind of restrictable plan (one
tile per transform, the four-step, the real pre/post four-step, pulse
compression in one tile and above it) the first `rows` outputs of a
row-limited exec must equal, bit for bit, those of the full exec of the same
plan (the same kernels run the same tiles), the rows after them must stay
untouched, and the result must match the FP64 oracle.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import random_input, settle, shapes

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-6

# (type, direction, n, plan batch, pulse)
CASES = [(O.C2C, O.FORWARD, 4096, 300, False), (O.C2C, O.INVERSE, 1000, 64, False),
         (O.C2C, O.FORWARD, 65536, 24, False), (O.R2C, O.FORWARD, 1 << 20, 6, False),
         (O.C2R, O.INVERSE, 1 << 20, 6, False), (O.R2C, O.FORWARD, 6000, 40, False),
         (O.C2C, O.FORWARD, 4096, 48, True), (O.C2C, O.FORWARD, 32768, 12, True)]


@pytest.mark.parametrize("typ,direction,n,batch,pulse", CASES)
def test_rows_exec_matches_full_exec(cuda, typ, direction, n, batch, pulse):
    from sip_b200.fft import FftHandle, check

    torch = cuda
    s = torch.cuda.Stream()
    h = FftHandle()
    filt = None
    if pulse:
        filt = torch.from_numpy(O.chirp_spectrum(n).astype(np.complex64)).cuda()
        check(h.make_plan_pulse_1d(n, batch, filt.data_ptr(), L.SIP_FFT_PULSE_CONJ_FILTER), "pulse plan")
    else:
        check(h.make_plan_1d(n, typ, direction, batch), "plan")
    check(h.set_stream(s), "stream")
    ws_size = h.workspace_size()
    check(ws_size[0], "workspace size")
    ws = torch.empty(max(1, ws_size[1]), dtype=torch.uint8, device="cuda")
    x = random_input(typ, [n], batch, seed=n + batch)
    _, _, oshape, odt = shapes(typ, [n], batch)
    tdt = torch.complex64 if odt == np.complex64 else torch.float32
    xt = torch.from_numpy(x).cuda()
    full = torch.zeros(oshape, dtype=tdt, device="cuda")
    settle()
    check(h.exec_rows(batch, xt.data_ptr(), full.data_ptr(), ws.data_ptr()), "full exec")
    s.synchronize()
    want_full = full.cpu().numpy()
    for rows in sorted({1, 5, batch // 2 + 1, batch}):
        if rows > batch:
            continue
        out = torch.full(oshape, 7.0, dtype=tdt, device="cuda")
        settle()
        check(h.exec_rows(rows, xt.data_ptr(), out.data_ptr(), ws.data_ptr()), f"rows={rows}")
        s.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got[:rows], want_full[:rows], err_msg=f"rows={rows}")
        assert (got[rows:] == 7.0).all(), f"rows={rows}: rows after the limit were written"
    if pulse:
        want = O.pulse(x[:2], filt.cpu().numpy(), conj=True)
    elif typ == O.C2R:
        want = np.fft.irfft(x[:2].astype(np.complex128), n=n, axis=-1) * n
    else:
        want = O.fp64(typ, direction, x[:2], [n])
    assert O.rel_l2(want_full[:2], want) <= REL_L2_TOL
    h.destroy()

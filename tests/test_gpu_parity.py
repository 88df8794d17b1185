"""Parity of the CUDA path with the oracle on a B200, through the C ABI.

Every reference unit-test case (tests/ref_cases.py) runs with the
reference's own inputs (fixed-seed LCG) and passes the reference's check:
numpy.fft golden in complex64 / float32, isclose(rtol=1e-3, atol=1e-5)
(absolute tolerance floored at 1e-6 of the peak, oracle.ref_check_mismatches).
Each case is also held to rel-L2 <= 1e-6 against the FP64 oracle, the
accuracy bar of this library.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import ref_cases as RC
from tests.fftcase import gpu_run, shapes

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-6


def _check(torch, op, direction, sizes, batch, record=None):
    ishape, idt, _, _ = shapes(op, sizes, batch)
    x = O.ut_input(ishape, idt)
    out = gpu_run(torch, op, direction, sizes, batch, x)
    gold = O.golden(op, direction, x, sizes)
    bad = O.ref_check_mismatches(out, gold)
    # the bins that meet the reference's isclose(1e-3, 1e-5) only with the
    # absolute tolerance floored at 1e-6 of the peak (near-zero bins of long
    # FP32 transforms): recorded per case (junit property
    # "isclose_floor_bins") and named in the failure message
    strict = O.isclose_mismatches(out, gold, 1e-3, 1e-5)
    if record is not None:
        record("isclose_floor_bins", strict - bad)
    err = O.rel_l2(out, O.fp64(op, direction, x, sizes))
    assert bad == 0, f"{bad} elements outside isclose(1e-3, 1e-5); rel_l2={err:.3e}"
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}; {strict} bins needed the floored atol"


@pytest.mark.parametrize("batch,n,direction", RC.C2C_1D)
def test_ref_c2c_1d(cuda, record_property, batch, n, direction):
    _check(cuda, O.C2C, direction, [n], batch, record_property)


@pytest.mark.parametrize("batch,n,direction", RC.R2C_1D)
def test_ref_r2c_1d(cuda, record_property, batch, n, direction):
    _check(cuda, O.R2C, direction, [n], batch, record_property)


@pytest.mark.parametrize("batch,n,direction", RC.C2R_1D)
def test_ref_c2r_1d(cuda, record_property, batch, n, direction):
    _check(cuda, O.C2R, direction, [n], batch, record_property)


@pytest.mark.parametrize("x,y,batch,direction", RC.C2C_2D)
def test_ref_c2c_2d(cuda, record_property, x, y, batch, direction):
    _check(cuda, O.C2C, direction, [x, y], batch, record_property)


@pytest.mark.parametrize("x,y,z,batch,direction", RC.C2C_3D)
def test_ref_c2c_3d(cuda, record_property, x, y, z, batch, direction):
    _check(cuda, O.C2C, direction, [x, y, z], batch, record_property)


# Real multi-dimensional transforms (R2C/C2R along the last axis, C2C on the others).
@pytest.mark.parametrize("op", [O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
@pytest.mark.parametrize("sizes,batch", [([64, 64], 1), ([32, 48], 2), ([500, 50], 2), ([30, 33], 3),
                                         ([8, 8, 8], 1), ([16, 12, 10], 2), ([9, 7, 5], 2)])
def test_real_multid(cuda, op, direction, sizes, batch):
    _check(cuda, op, direction, sizes, batch)


@pytest.mark.parametrize("pattern", ["zero", "constant", "impulse", "nyquist", "random"])
@pytest.mark.parametrize("op", [O.C2C, O.R2C, O.C2R])
@pytest.mark.parametrize("n", [64, 1000, 4096])
def test_known_answers(cuda, pattern, op, n):
    """Known-answer patterns of tests/standalone/fft1d_optimized/run.py:61-107 (FP64 golden, rel-L2)."""
    for direction in (O.FORWARD, O.INVERSE):
        x, g = O.kat_input(pattern, op, n, 4, 1, direction)
        out = gpu_run(cuda, op, direction, [n], 4, x)
        assert np.isfinite(out).all()
        if np.linalg.norm(g) == 0:
            assert np.abs(out).max() == 0
        else:
            assert O.rel_l2(out, g) <= REL_L2_TOL


# Every size-specialized kernel with more tiles than resident CTAs, so each
# CTA transforms several tiles and the double-buffered staging of the next
# tile runs (grids are capped at SMs x resident CTAs; 148 x 3 = 444 for the
# smaller kernels).
@pytest.mark.parametrize("op,direction,n,batch", [
    (O.C2C, O.FORWARD, 4096, 1000), (O.C2C, O.INVERSE, 4096, 1000),
    (O.C2C, O.FORWARD, 8192, 700), (O.C2C, O.INVERSE, 8192, 700),
    (O.C2C, O.FORWARD, 2048, 2000), (O.C2C, O.INVERSE, 1024, 4000),
    (O.C2C, O.FORWARD, 256, 16000),
    (O.C2C, O.FORWARD, 65536, 300), (O.C2C, O.INVERSE, 524288, 40),
    (O.R2C, O.FORWARD, 1000, 8000), (O.C2R, O.INVERSE, 1000, 8000),
    (O.R2C, O.FORWARD, 6000, 2000), (O.C2R, O.INVERSE, 6000, 2000),
    (O.R2C, O.FORWARD, 2187, 2001), (O.C2R, O.INVERSE, 2187, 2001),
    (O.R2C, O.FORWARD, 1 << 20, 12), (O.C2R, O.INVERSE, 1 << 20, 12),
])
def test_specialized_kernels_many_tiles_per_cta(cuda, op, direction, n, batch):
    rng = np.random.default_rng(n + batch)
    ishape, idt, _, _ = shapes(op, [n], batch)
    if idt == np.float32:
        x = rng.uniform(-1, 1, ishape).astype(np.float32)
    else:
        x = (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64)
    out = gpu_run(cuda, op, direction, [n], batch, x)
    rows = np.unique(np.linspace(0, batch - 1, 24).astype(np.int64))
    err = O.rel_l2(out[rows], O.fp64(op, direction, x[rows], [n]))
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}"


# Both forms of the large real transforms (fused mirrored passes, or the
# plain four-step plus a pre/post pass), selected with the planner hint.
@pytest.mark.parametrize("op,direction", [(O.R2C, O.FORWARD), (O.C2R, O.INVERSE), (O.R2C, O.INVERSE),
                                          (O.C2R, O.FORWARD)])
@pytest.mark.parametrize("fused", [1, 2])
def test_large_real_forms(cuda, op, direction, fused):
    from sip_b200 import _lib as L
    from sip_b200.fft import FftHandle, check
    from tests.fftcase import settle

    n, batch = 1 << 20, 3
    ishape, idt, oshape, odt = shapes(op, [n], batch)
    rng = np.random.default_rng(fused)
    x = (rng.uniform(-1, 1, ishape).astype(np.float32) if idt == np.float32 else
         (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64))
    xt = cuda.from_numpy(x).cuda()
    yt = cuda.zeros(oshape, dtype=cuda.complex64 if odt == np.complex64 else cuda.float32, device="cuda")
    h = FftHandle()
    check(h.set_hint(L.SIP_FFT_HINT_REAL_FUSED, fused), "hint")
    check(h.make_plan_1d(n, op, direction, batch), "plan")
    h.bind_workspace()
    s = cuda.cuda.Stream()
    check(h.set_stream(s), "stream")
    settle()
    check((h.exec_r2c if op == O.R2C else h.exec_c2r)(xt, yt), "exec")
    s.synchronize()
    assert O.rel_l2(yt.cpu().numpy(), O.fp64(op, direction, x, [n])) <= REL_L2_TOL
    h.destroy()


# Lengths whose factors include the prime radices 23, 29 and 31, planned
# as direct passes: 2^7 23, 2^5 3 31, 2^6 29, 31^2, 23 29, and 23 31 29 2^2
# above one tile.
@pytest.mark.parametrize("n,batch", [(2944, 40), (2976, 40), (1856, 33), (961, 17), (667, 9), (82708, 3)])
@pytest.mark.parametrize("op", [O.C2C, O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_prime_radix_lengths(cuda, n, batch, op, direction):
    rng = np.random.default_rng(n + 7 * op)
    ishape, idt, _, _ = shapes(op, [n], batch)
    if op == O.C2R:
        x = np.fft.rfft(rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
    elif idt == np.float32:
        x = rng.uniform(-1, 1, ishape).astype(np.float32)
    else:
        x = (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64)
    out = gpu_run(cuda, op, direction, [n], batch, x)
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}"


# Lengths with a prime factor above 32: Bluestein (pre pass, fused
# convolution of a 2,3,5-smooth length, post pass).
@pytest.mark.parametrize("n,batch", [(41, 5), (37, 64), (1009, 33), (4099, 7), (2 * 8191, 5), (20011, 3),
                                     (65537, 2)])
@pytest.mark.parametrize("op", [O.C2C, O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_bluestein_lengths(cuda, n, batch, op, direction):
    rng = np.random.default_rng(n + op)
    ishape, idt, _, _ = shapes(op, [n], batch)
    if op == O.C2R:
        x = np.fft.rfft(rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
    elif idt == np.float32:
        x = rng.uniform(-1, 1, ishape).astype(np.float32)
    else:
        x = (rng.standard_normal(ishape) + 1j * rng.standard_normal(ishape)).astype(np.complex64)
    out = gpu_run(cuda, op, direction, [n], batch, x)
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"rel_l2 vs FP64 {err:.3e}"


@pytest.mark.parametrize("op,direction,n,batch", [(O.C2C, O.FORWARD, (1 << 22) + 1, 2),
                                                   (O.C2C, O.INVERSE, 5000011, 1),
                                                   (O.R2C, O.FORWARD, 2 * 4194319, 1)])
def test_bluestein_above_2p22(cuda, op, direction, n, batch):
    """Lengths with a large prime factor above 2^22: the convolution is longer
    than the host's FP64 filter transform handles quickly, so its filter is
    the library's own FP32 transform of the FP64-made sequence, on the GPU."""
    from tests.fftcase import random_input

    x = random_input(op, [n], batch, seed=n % 1000)
    out = gpu_run(cuda, op, direction, [n], batch, x)
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"n={n}: rel_l2 {err:.3e}"


@pytest.mark.parametrize("n", [59049, 98415, 177147])
@pytest.mark.parametrize("op,direction", [(O.R2C, O.FORWARD), (O.R2C, O.INVERSE), (O.C2R, O.INVERSE),
                                          (O.C2R, O.FORWARD)])
@pytest.mark.parametrize("batch", [1, 6, 7])
def test_odd_real_above_one_tile(cuda, n, op, direction, batch):
    """Odd real lengths above one tile (3^10, 3^9 5, 3^11): row pairs through
    the complex four-step, as the reference's arch35 real core takes them."""
    from tests.fftcase import random_input

    x = random_input(op, [n], batch, seed=n + batch)
    out = gpu_run(cuda, op, direction, [n], batch, x)
    err = O.rel_l2(out, O.fp64(op, direction, x, [n]))
    assert err <= REL_L2_TOL, f"n={n} batch={batch}: rel_l2 {err:.3e}"


@pytest.mark.parametrize("n,batch", [(1024, 1024), (4096, 256), (8192, 3), (4096, 1)])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_cluster_four_step(cuda, n, batch, direction, monkeypatch):
    """With SIP_FFT_CLUSTER=1, small C2C batches run one transform per
    thread-block cluster (the CTAs exchanging through distributed shared
    memory); by default the same plan runs the one-CTA-per-transform
    kernel.  Both match FP64."""
    from tests.fftcase import random_input
    from sip_b200.fft import FftHandle

    x = random_input(O.C2C, [n], batch, seed=n + batch)
    want = O.fp64(O.C2C, direction, x, [n])
    monkeypatch.setenv("SIP_FFT_CLUSTER", "1")
    h = FftHandle()
    assert h.make_plan_1d(n, O.C2C, direction, batch) == 0
    assert h.describe()["steps"][0]["kind"] == 9   # the cluster step
    h.destroy()
    out = gpu_run(cuda, O.C2C, direction, [n], batch, x)
    assert O.rel_l2(out, want) <= REL_L2_TOL
    monkeypatch.delenv("SIP_FFT_CLUSTER")
    h = FftHandle()
    assert h.make_plan_1d(n, O.C2C, direction, batch) == 0
    assert h.describe()["steps"][0]["kind"] != 9
    h.destroy()
    out0 = gpu_run(cuda, O.C2C, direction, [n], batch, x)
    assert O.rel_l2(out0, want) <= REL_L2_TOL


# (type, direction, planner hints, step holding the mirrored pairs, its length)
MIRRORED_FORMS = [
    (O.R2C, O.FORWARD, {}, 1, 512),             # default: 1024 x 512 split, pass B on pairs
    (O.R2C, O.INVERSE, {}, 1, 512),
    (O.R2C, O.FORWARD, {6: 2}, 1, 1024),        # 512 x 1024 split, pass B on pairs (variant)
    (O.C2R, O.INVERSE, {5: 1, 6: 1}, 0, 512),   # fused pre-process in pass A on pairs (variant)
    (O.C2R, O.FORWARD, {5: 1, 6: 1}, 0, 512),
    (O.C2R, O.INVERSE, {5: 1, 6: 0}, 0, None),  # fused pre-process, element by element (variant)
]


@pytest.mark.parametrize("op,direction,hints,step,n_pair", MIRRORED_FORMS)
@pytest.mark.parametrize("batch", [1, 5])
def test_real_four_step_mirrored_forms(cuda, op, direction, hints, step, n_pair, batch):
    """The real 2^20 four-step forms whose pass B (R2C) or pass A (C2R)
    handles a row or column together with its mirror: the planner picks the
    expected kernel (TWB bit 4 where the post- or pre-process runs on
    mirrored butterfly pairs) and the result matches FP64."""
    from tests.fftcase import random_input, settle, shapes
    from sip_b200.fft import FftHandle, check

    torch = cuda
    n = 1 << 20
    x = random_input(op, [n], batch, seed=batch + 31 * len(hints))
    h = FftHandle()
    for k, v in hints.items():
        check(h.set_hint(k, v), "hint")
    check(h.make_plan_1d(n, op, direction, batch), "plan")
    cfg = h.describe()["steps"][step]["sk_cfg"]
    if n_pair is None:
        assert not cfg[8] & 4
    else:
        assert cfg[8] & 4 and cfg[0] == n_pair, cfg
    h.bind_workspace()
    s = torch.cuda.Stream()
    check(h.set_stream(s), "stream")
    _, _, oshape, odt = shapes(op, [n], batch)
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yt = torch.zeros(oshape, dtype=torch.complex64 if odt == np.complex64 else torch.float32, device="cuda")
    settle()
    check((h.exec_r2c if op == O.R2C else h.exec_c2r)(xt, yt), "exec")
    s.synchronize()
    err = O.rel_l2(yt.cpu().numpy(), O.fp64(op, direction, x, [n]))
    h.destroy()
    assert err <= REL_L2_TOL, f"rel_l2 {err:.3e}"


# Multi-dimensional C2C whose contiguous last axis is above one tile (the
# batched 1-D four-step of the rows) or needs Bluestein (prime 20011, and
# 2053 whose convolution fits one tile), then the column passes.
@pytest.mark.parametrize("sizes,batch", [([4, 20011], 2), ([3, 5, 2053], 2), ([6, 40000], 2),
                                         ([2, 3, 65536], 1), ([24, 131072], 1)])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_multid_large_or_bluestein_last_axis(cuda, sizes, batch, direction):
    _check(cuda, O.C2C, direction, sizes, batch)


# Multi-dimensional real plans whose last axis is above one tile (even, and
# odd 59049 = 3^10 through row pairs).
@pytest.mark.parametrize("sizes,batch", [([3, 40000], 2), ([2, 3, 65536], 1), ([12, 1 << 20], 1), ([5, 59049], 2)])
@pytest.mark.parametrize("op", [O.R2C, O.C2R])
@pytest.mark.parametrize("direction", [O.FORWARD, O.INVERSE])
def test_multid_real_large_last_axis(cuda, sizes, batch, op, direction):
    _check(cuda, op, direction, sizes, batch)

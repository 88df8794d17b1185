"""Serving loop on the GPU: every request's result is the same in the mix as
alone (bitwise, same kernels), matches the plain per-request FP32 path
within tolerance, and matches the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from sip_b200.serve import (KIND_PULSE, PlainExecutor, QueueExecutor, Request, Scheduler, make_requests)

pytestmark = pytest.mark.gpu

REL_L2_TOL = 1e-6


def want(r, x):
    if r.kind == KIND_PULSE:
        return O.pulse(x, O.chirp_spectrum(r.n), conj=True)
    return np.fft.fft(x.astype(np.complex128), axis=-1)


def test_serving_mix_equals_alone_and_plain(cuda):
    torch = cuda
    reqs = make_requests(40, rate_hz=float("inf"), seed=11, lo=256, hi=1 << 17, max_batch=24, fft_share=0.3)
    lengths = sorted({r.n for r in reqs})
    budget = 160 << 20  # smaller than the whole set: admission has to wait for completions
    ex = QueueExecutor(torch, budget, lengths, max_batch=24, streams=2)
    saved = {}

    def keep(group):
        for r in group:
            saved[r.rid] = (ex.input(r).clone(), ex.output(r).clone())

    stats = Scheduler(ex, budget, max_inflight=2, on_complete=keep).run(reqs)
    assert len(stats.requests) == len(reqs) and stats.max_group > 1 and stats.groups > 1
    assert stats.peak_bytes <= budget

    pl = PlainExecutor(torch, budget)
    for r in reqs:
        x, y = saved[r.rid]
        alone = Request(r.rid, r.kind, r.n, r.batch, 0.0, r.delay)
        got = {}
        ex.fixed[r.rid] = x
        Scheduler(ex, budget, on_complete=lambda g: got.update({q.rid: ex.output(q).clone() for q in g})).run([alone])
        assert torch.equal(got[r.rid], y), (r.kind, r.n, r.batch)
        plain = Request(r.rid, r.kind, r.n, r.batch, 0.0, r.delay)
        pl.fixed[r.rid] = x
        pgot = {}
        Scheduler(pl, budget, max_group=1,
                  on_complete=lambda g: pgot.update({q.rid: pl.output(q).clone() for q in g})).run([plain])
        xh, yh, ph = x.cpu().numpy(), y.cpu().numpy(), pgot[r.rid].cpu().numpy()
        w = want(r, xh)
        assert O.rel_l2(yh, w) <= REL_L2_TOL, (r.kind, r.n, r.batch)
        assert O.rel_l2(ph, w) <= REL_L2_TOL
        assert O.rel_l2(yh, ph) <= 2 * REL_L2_TOL
    ex.close()
    pl.close()


def test_serving_latency_stats(cuda):
    torch = cuda
    reqs = make_requests(200, rate_hz=2000.0, seed=12, lo=256, hi=1 << 16, max_batch=64)
    budget = 1 << 30
    ex = QueueExecutor(torch, budget, sorted({r.n for r in reqs}), max_batch=64)
    s = Scheduler(ex, budget).run(reqs).summary()
    assert s["requests"] == 200 and 0 < s["p50_ms"] <= s["p99_ms"]
    assert all(r.done >= r.arrival for r in reqs)
    ex.close()


def test_resident_executor_mix_equals_alone(cuda):
    """The resident executor (specialized kernels, one row-limited exec per
    request): each request's result is the same in the mix as alone and
    matches the FP64 oracle."""
    from sip_b200.serve import ResidentExecutor

    torch = cuda
    reqs = make_requests(30, rate_hz=float("inf"), seed=13, lo=256, hi=1 << 17, max_batch=24, fft_share=0.3)
    lengths = sorted({r.n for r in reqs})
    budget = 160 << 20
    ex = ResidentExecutor(torch, budget, lengths, max_batch=24, streams=2)
    saved = {}

    def keep(group):
        for r in group:
            saved[r.rid] = (ex.input(r).clone(), ex.output(r).clone())

    stats = Scheduler(ex, budget, max_inflight=2, on_complete=keep).run(reqs)
    assert len(stats.requests) == len(reqs) and stats.max_group > 1
    for r in reqs:
        x, y = saved[r.rid]
        alone = Request(r.rid, r.kind, r.n, r.batch, 0.0, r.delay)
        got = {}
        ex.fixed[r.rid] = x
        Scheduler(ex, budget, on_complete=lambda g: got.update({q.rid: ex.output(q).clone() for q in g})).run([alone])
        assert torch.equal(got[r.rid], y), (r.kind, r.n, r.batch)
        assert O.rel_l2(y.cpu().numpy(), want(r, x.cpu().numpy())) <= REL_L2_TOL, (r.kind, r.n, r.batch)
    ex.close()

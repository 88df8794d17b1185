"""Serving loop logic on the CPU: request generation, the arena, and the
scheduler's admission and continuous grouping, driven by a fake clock and a
fake executor whose groups take a modelled service time."""
import math

import numpy as np
import pytest

from sip_b200.serve import KIND_FFT, KIND_PULSE, Arena, Request, Scheduler, make_requests, smooth_lengths


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class FakeExecutor:
    """One device: a group occupies it for the sum of its requests' service
    times (bytes / 4 TB/s + 5 us), in launch order."""

    def __init__(self, clock):
        self.clock = clock
        self.busy_until = 0.0
        self.launched = []
        self.finished = []

    def bytes_needed(self, r):
        return 2 * r.batch * r.n * 8

    def start(self):
        pass

    def now(self):
        return self.clock.t

    def launch(self, group):
        self.launched.append([r.rid for r in group])
        start = max(self.clock.t, self.busy_until)
        self.busy_until = start + sum(self.bytes_needed(r) / 4e12 + 5e-6 for r in group)
        return self.busy_until

    def poll(self, token):
        return token if self.clock.t >= token else None

    def finish(self, group):
        self.finished.extend(r.rid for r in group)


def run(reqs, budget=1 << 34, inflight=2, group=256):
    clk = FakeClock()
    ex = FakeExecutor(clk)
    sch = Scheduler(ex, budget, max_inflight=inflight, max_group=group, sleep=clk.sleep)
    return sch.run(reqs), ex


def test_smooth_lengths():
    lens = smooth_lengths(256, 1 << 18)
    assert lens[0] == 256 and lens[-1] == 1 << 18
    for n in lens:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        assert m == 1
    assert 1000 in lens and 2187 in lens and 6000 in lens and 1001 not in lens


def test_make_requests_distribution():
    reqs = make_requests(4000, rate_hz=1e4, seed=1, fft_share=0.25)
    n = np.array([r.n for r in reqs])
    b = np.array([r.batch for r in reqs])
    t = np.array([r.arrival for r in reqs])
    assert n.min() >= 256 and n.max() <= 1 << 18
    assert b.min() >= 1 and b.max() <= 512 and abs(b.mean() - 256.5) < 15
    assert np.all(np.diff(t) >= 0) and abs(len(t) / t[-1] - 1e4) / 1e4 < 0.1  # Poisson rate
    mid = math.log(256 * (1 << 18)) / 2                                     # log-uniform median
    assert abs(np.median(np.log(n)) - mid) < 0.5
    assert 0.2 < np.mean([r.kind == KIND_FFT for r in reqs]) < 0.3
    assert all(0 <= r.delay <= r.n - max(1, r.n // 4) for r in reqs)
    again = make_requests(4000, rate_hz=1e4, seed=1, fft_share=0.25)
    assert [(r.n, r.batch, r.arrival) for r in again] == [(r.n, r.batch, r.arrival) for r in reqs]


def test_arena_first_fit_and_merge():
    a = Arena(4096)
    x = a.alloc(1000)
    y = a.alloc(1000)
    z = a.alloc(1000)
    assert (x, y, z) == (0, 1024, 2048)
    assert a.alloc(2000) is None
    a.release(y)
    assert a.alloc(1024) == 1024
    a.release(1024)
    a.release(x)
    a.release(z)
    assert a.free == [(0, 4096)] and a.in_use == 0


def test_every_request_completes_in_fifo_order():
    reqs = make_requests(500, rate_hz=2e4, seed=3)
    stats, ex = run(reqs)
    assert len(stats.requests) == 500
    order = [rid for g in ex.launched for rid in g]
    assert order == sorted(order)                      # FIFO admission and launch
    for r in stats.requests:
        assert r.done >= r.launched >= r.arrival
        assert r.latency > 0


def test_continuous_batching_groups_concurrent_arrivals():
    reqs = [Request(i, KIND_PULSE, 4096, 64, 0.0) for i in range(100)]
    stats, ex = run(reqs, inflight=1)
    assert stats.groups < 100 and stats.max_group > 1
    assert len(ex.launched[0]) == 100                   # all arrived before the first launch


def test_admission_respects_budget():
    reqs = [Request(i, KIND_PULSE, 16384, 100, 0.0) for i in range(20)]
    need = 2 * 16384 * 100 * 8
    stats, ex = run(reqs, budget=3 * need, inflight=4)
    assert stats.peak_bytes <= 3 * need
    assert max(len(g) for g in ex.launched) <= 3
    assert len(stats.requests) == 20


def test_request_larger_than_budget_is_rejected():
    with pytest.raises(ValueError):
        run([Request(0, KIND_PULSE, 1 << 18, 512, 0.0)], budget=1 << 20)


def test_summary_fields():
    stats, _ = run(make_requests(50, rate_hz=1e3, seed=5))
    s = stats.summary()
    assert s["requests"] == 50 and s["p99_ms"] >= s["p50_ms"] > 0 and s["throughput_req_s"] > 0

"""Continuous-batching serving loop for FFT and pulse-compression requests.

Requests (FFT, or pulse compression = FFT, multiply by the conjugate
spectrum of the transmitted chirp, IFFT) of mixed lengths and batch counts
arrive over time.  The loop admits each arrival as soon as its memory fits
the HBM admission budget, and launches everything admitted but not yet
launched as ONE group while fewer than `max_inflight` groups are on the GPU,
so requests that arrive while others run join the next group and their work
overlaps on the device.  Plans, twiddle tables and filter spectra stay
resident; each request's input, output and workspace come from one arena
sized to the budget.

Three executors share the scheduler:
  * `QueueExecutor`: the library's persistent work queue (sipFftBatch*), one
    launch per pass index for the whole group, replayed from a captured CUDA
    graph, with the fused pulse-compression kernels; one plan per length
    (batch 512) serves any batch through sipFftBatchAddRows.
  * `ResidentExecutor`: the same resident plans (one per length, batch
    512) on the size-specialized and run-time compiled kernels instead of
    the queue's generic tile body; every request of a group runs its rows
    through its length's plan (sipFftExecRawRows), the group's launches on
    one of several streams (launches of consecutive requests overlap through
    programmatic dependent launch).
  * `PlainExecutor`: the plain per-request FP32 path, as a user of the
    reference's API writes it: per request a forward C2C exec, an
    elementwise multiply, an inverse C2C exec, with plans kept in an LRU
    cache of 10 (N, batch) entries like sip_pta's FFTMixCache.

Completion times are device times (CUDA events against an event recorded
when the run starts), so latency = completion - arrival on one clock.
The scheduler itself takes a clock, a sleep and an executor interface, so
its admission and grouping logic is tested on the CPU with a fake clock.
"""
from __future__ import annotations

import bisect
import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

KIND_PULSE = "pulse"
KIND_FFT = "fft"


@dataclass
class Request:
    rid: int
    kind: str
    n: int
    batch: int
    arrival: float          # seconds from the start of the run
    delay: int = 0          # chirp delay of the synthetic signal
    offset: int = -1        # arena offset while admitted
    launched: float = math.nan
    done: float = math.nan  # device completion time, seconds from the start

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def smooth_lengths(lo: int = 256, hi: int = 1 << 18) -> list[int]:
    """Every 2^a 3^b 5^c in [lo, hi], ascending."""
    out = set()
    p2 = 1
    while p2 <= hi:
        p3 = p2
        while p3 <= hi:
            p5 = p3
            while p5 <= hi:
                if p5 >= lo:
                    out.add(p5)
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def make_requests(count: int, rate_hz: float, seed: int = 20261203, lo: int = 256, hi: int = 1 << 18,
                  max_batch: int = 512, fft_share: float = 0.0) -> list[Request]:
    """Poisson arrivals at `rate_hz` (all at t=0 when rate_hz is inf); N
    log-uniform over the 2,3,5-smooth lengths in [lo, hi] (a log-uniform draw
    rounded up to the next smooth length); batch uniform in 1..max_batch;
    a share `fft_share` of plain forward-FFT requests, the rest pulse
    compression."""
    rng = np.random.default_rng(seed)
    lens = smooth_lengths(lo, hi)
    t = 0.0
    out = []
    for i in range(count):
        if math.isfinite(rate_hz):
            t += float(rng.exponential(1.0 / rate_hz))
        x = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        n = lens[min(bisect.bisect_left(lens, x), len(lens) - 1)]
        b = int(rng.integers(1, max_batch + 1))
        kind = KIND_FFT if rng.random() < fft_share else KIND_PULSE
        L = max(1, n // 4)
        out.append(Request(i, kind, n, b, t, delay=int(rng.integers(0, n - L + 1))))
    return out


def request_flops(r: Request) -> float:
    f = 5.0 * r.n * math.log2(r.n) * r.batch
    return 2 * f + 6.0 * r.n * r.batch if r.kind == KIND_PULSE else f


class Arena:
    """First-fit allocator of byte ranges in [0, capacity) (256-byte aligned)."""

    ALIGN = 256

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        self.free = [(0, self.capacity)]  # sorted (offset, size)
        self.used = {}

    def alloc(self, size: int):
        size = (int(size) + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        for i, (off, sz) in enumerate(self.free):
            if sz >= size:
                if sz == size:
                    del self.free[i]
                else:
                    self.free[i] = (off + size, sz - size)
                self.used[off] = size
                return off
        return None

    def release(self, off: int) -> None:
        size = self.used.pop(off)
        i = bisect.bisect_left(self.free, (off, 0))
        self.free.insert(i, (off, size))
        # merge with neighbours
        if i + 1 < len(self.free) and off + size == self.free[i + 1][0]:
            self.free[i] = (off, size + self.free[i + 1][1])
            del self.free[i + 1]
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == self.free[i][0]:
            self.free[i - 1] = (self.free[i - 1][0], self.free[i - 1][1] + self.free[i][1])
            del self.free[i]

    @property
    def in_use(self) -> int:
        return sum(self.used.values())


@dataclass
class RunStats:
    requests: list = field(default_factory=list)
    makespan: float = 0.0
    groups: int = 0
    peak_bytes: int = 0
    max_group: int = 0

    def summary(self) -> dict:
        lat = np.array([r.latency for r in self.requests]) * 1e3
        flops = sum(request_flops(r) for r in self.requests)
        return {
            "requests": len(self.requests),
            "p50_ms": round(float(np.percentile(lat, 50)), 4),
            "p99_ms": round(float(np.percentile(lat, 99)), 4),
            "mean_ms": round(float(lat.mean()), 4),
            "throughput_req_s": round(len(self.requests) / self.makespan, 2),
            "gflops": round(flops / self.makespan / 1e9, 2),
            "makespan_s": round(self.makespan, 4),
            "groups": self.groups,
            "max_group": self.max_group,
            "peak_arena_gb": round(self.peak_bytes / 1e9, 3),
        }


class Scheduler:
    """Admission against the arena budget and continuous grouping.

    executor interface: bytes_needed(r), start(), launch(group) -> token,
    poll(token) -> device completion time (s) or None, finish(group), and
    `now()` for the current time on the device clock."""

    def __init__(self, executor, budget_bytes: int, max_inflight: int = 3, max_group: int = 256,
                 sleep=time.sleep, on_complete=None):
        self.ex = executor
        self.arena = Arena(budget_bytes)
        self.max_inflight = max_inflight
        self.max_group = max_group
        self.sleep = sleep
        self.on_complete = on_complete

    def run(self, requests) -> RunStats:
        ex = self.ex
        for r in requests:
            if ex.bytes_needed(r) > self.arena.capacity:
                raise ValueError(f"request {r.rid} needs more than the whole budget")
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        admitted = []
        inflight = []
        stats = RunStats()
        ex.start()
        while pending or waiting or admitted or inflight:
            now = ex.now()
            progressed = False
            for item in list(inflight):
                token, group = item
                t = ex.poll(token)
                if t is None:
                    continue
                inflight.remove(item)
                for r in group:
                    r.done = t
                if self.on_complete is not None:
                    self.on_complete(group)
                ex.finish(group)
                for r in group:
                    self.arena.release(r.offset)
                    r.offset = -1
                    stats.requests.append(r)
                progressed = True
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while waiting:  # FIFO admission: no request overtakes an earlier one
                off = self.arena.alloc(ex.bytes_needed(waiting[0]))
                if off is None:
                    break
                r = waiting.popleft()
                r.offset = off
                admitted.append(r)
                progressed = True
            stats.peak_bytes = max(stats.peak_bytes, self.arena.in_use)
            if admitted and len(inflight) < self.max_inflight:
                group, admitted = admitted[:self.max_group], admitted[self.max_group:]
                for r in group:
                    r.launched = now
                inflight.append((ex.launch(group), group))
                stats.groups += 1
                stats.max_group = max(stats.max_group, len(group))
                continue
            if not progressed:
                nxt = pending[0].arrival - now if pending else 0.0
                self.sleep(max(0.0, min(nxt, 20e-6)) if inflight or not pending else max(0.0, min(nxt, 1e-3)))
        scale = getattr(ex, "clock_scale", None)
        if callable(scale):  # device completion times onto the host clock
            s = scale()
            for r in stats.requests:
                r.done *= s
        stats.makespan = max(r.done for r in stats.requests) - min(r.arrival for r in stats.requests)
        return stats


# --------------------------------------------------------------- executors
class _GpuBase:
    """Arena memory, synthetic signals and the device clock."""

    def __init__(self, torch, budget_bytes: int, device=None):
        self.torch = torch
        self.dev = torch.device(device or "cuda")
        self.mem = torch.empty(int(budget_bytes), dtype=torch.uint8, device=self.dev)
        self.base = self.mem.data_ptr()
        self.chirps = {}
        self.filters = {}
        self.gen = torch.Generator(device=self.dev)
        self.gen.manual_seed(20261203)
        self.t0_event = None
        self.fixed = {}  # rid -> device tensor used as the input instead of a generated signal

    @staticmethod
    def needs_ws(r: Request) -> bool:
        return r.n > 16384

    def regions(self, r: Request):
        """Arena offsets of the request's input, output and workspace."""
        per = r.batch * r.n * 8
        step = (per + Arena.ALIGN - 1) // Arena.ALIGN * Arena.ALIGN
        return r.offset, r.offset + step, (r.offset + 2 * step if self.needs_ws(r) else None)

    def bytes_needed(self, r: Request) -> int:
        per = (r.batch * r.n * 8 + Arena.ALIGN - 1) // Arena.ALIGN * Arena.ALIGN
        return per * (3 if self.needs_ws(r) else 2)

    def output(self, r: Request):
        return self.view(self.regions(r)[1], r.batch * r.n).view(r.batch, r.n)

    def input(self, r: Request):
        return self.view(self.regions(r)[0], r.batch * r.n).view(r.batch, r.n)

    def view(self, off: int, count: int):
        """complex64 tensor of `count` values at arena offset `off`."""
        return self.mem[off:off + count * 8].view(self.torch.complex64)

    def prepare_signals(self, lengths) -> None:
        """The transmitted chirp of every length, made before any timing:
        made on first use inside a run, its pageable host-to-device copy
        waits behind the work already queued on the stream."""
        for n in lengths:
            self.chirp(n)
        self.torch.cuda.synchronize(self.dev)

    def chirp(self, n: int):
        if n not in self.chirps:
            L = max(1, n // 4)
            t = np.arange(L)
            c = np.exp(1j * np.pi * t * t / L).astype(np.complex64)
            self.chirps[n] = self.torch.from_numpy(c).to(self.dev)
        return self.chirps[n]

    def filter(self, n: int):
        """Spectrum of the zero-padded chirp, once per length: the chirp is
        made on the device (FP64, rounded once) and transformed by the
        library's own forward C2C plan, on the GPU."""
        if n not in self.filters:
            from .fft import FftHandle, check
            from . import _lib as L

            torch = self.torch
            Lc = max(1, n // 4)
            t = torch.arange(Lc, dtype=torch.float64, device=self.dev)
            c = torch.zeros(n, dtype=torch.complex64, device=self.dev)
            c[:Lc] = torch.exp(1j * math.pi * t * t / Lc).to(torch.complex64)
            spec = torch.empty_like(c)
            torch.cuda.synchronize(self.dev)  # the chirp, made on torch's stream
            h = FftHandle()
            try:
                check(h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, 1), "filter plan")
                h.bind_workspace(self.dev)
                s = self.streams[0]
                check(h.set_stream(s), "filter stream")
                check(h.exec_raw(c.data_ptr(), spec.data_ptr()), "filter exec")
                s.synchronize()
            finally:
                h.destroy()
            self.filters[n] = spec
        return self.filters[n]

    def make_signal(self, r: Request, x) -> None:
        """Delayed chirp plus complex noise (sigma 0.1 per component), written
        on the current stream into the request's input region."""
        xv = x.view(r.batch, r.n)
        if r.rid in self.fixed:
            xv.copy_(self.fixed[r.rid])
            return
        self.torch.view_as_real(xv).normal_(0.0, 0.1, generator=self.gen)
        L = max(1, r.n // 4)
        xv[:, r.delay:r.delay + L] += self.chirp(r.n)

    def start(self) -> None:
        # The device is idle when the start event is recorded, so the event
        # runs within microseconds of the record call: the host clock is
        # read right before it, and host and device times share one origin
        # (device times are at most those microseconds late).
        self.torch.cuda.synchronize(self.dev)
        self.t0_event = self.torch.cuda.Event(enable_timing=True)
        self.t0_host = time.perf_counter()
        self.t0_event.record(self.streams[0])
        self.t0_event.synchronize()

    def now(self) -> float:
        return time.perf_counter() - self.t0_host

    def clock_scale(self) -> float:
        """Host seconds per device-timer second over the run: a second pair
        of host and device stamps at its end (the two clocks drift apart by
        about ten microseconds per second, which over a run of tens of
        seconds exceeds the latencies being measured).  Device completion
        times are multiplied by it."""
        torch = self.torch
        torch.cuda.synchronize(self.dev)
        t1 = torch.cuda.Event(enable_timing=True)
        t1_host = time.perf_counter()
        t1.record(self.streams[0])
        t1.synchronize()
        dev = self.t0_event.elapsed_time(t1) / 1e3
        return (t1_host - self.t0_host) / dev if dev > 0 else 1.0

    def poll(self, token):
        ev = token
        if not ev.query():
            return None
        return self.t0_event.elapsed_time(ev) / 1e3

    def finish(self, group) -> None:
        pass


class QueueExecutor(_GpuBase):
    """Groups through the persistent work queue with resident per-length plans."""

    def __init__(self, torch, budget_bytes: int, lengths, max_batch: int = 512, streams: int = 3,
                 use_graphs: bool = True, device=None):
        super().__init__(torch, budget_bytes, device)
        from . import _lib as L
        from .fft import Batch, FftHandle, check

        self.L = L
        self.check = check
        self.max_batch = max_batch
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(streams)]
        self.batches = [Batch(use_graphs) for _ in range(streams)]
        self.slot_event = [None] * streams
        self.next = 0
        self.plans = {}
        for n in lengths:
            for kind in (KIND_PULSE, KIND_FFT):
                h = FftHandle()
                check(h.set_hint(L.SIP_FFT_HINT_GENERIC_ONLY, 1), "hint")
                if kind == KIND_PULSE:
                    check(h.make_plan_pulse_1d(n, max_batch, self.filter(n).data_ptr(), L.SIP_FFT_PULSE_CONJ_FILTER),
                          "pulse plan")
                else:
                    check(h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, max_batch), "fft plan")
                self.plans[(kind, n)] = h
        self.prepare_signals(lengths)
        self.launches = 0

    def _free_slot(self) -> int:
        """A stream / batch slot whose last group has completed (a batch
        object's next exec waits for its previous one on the host), else the
        least recently used one."""
        for k in range(len(self.streams)):
            i = (self.next + k) % len(self.streams)
            ev = self.slot_event[i]
            if ev is None or ev.query():
                return i
        return self.next

    def launch(self, group):
        torch = self.torch
        i = self._free_slot()
        self.next = (i + 1) % len(self.streams)
        s = self.streams[i]
        bt = self.batches[i]
        check = self.check
        with torch.cuda.stream(s):
            for r in group:
                self.make_signal(r, self.view(self.regions(r)[0], r.batch * r.n))
        check(bt.clear(), "batch clear")
        for r in group:
            x, y, ws = self.regions(r)
            check(bt.add_rows(self.plans[(r.kind, r.n)], self.base + x, self.base + y, r.batch,
                              self.base + ws if ws is not None else None), "batch add rows")
        check(bt.execute(s), "batch exec")
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        self.slot_event[i] = ev
        self.launches += 1
        return ev

    def close(self) -> None:
        for b in self.batches:
            b.destroy()
        for h in self.plans.values():
            h.destroy()


class ResidentExecutor(_GpuBase):
    """Groups through resident per-length plans on the specialized kernels,
    one row-limited exec per request."""

    def __init__(self, torch, budget_bytes: int, lengths, max_batch: int = 512, streams: int = 4,
                 jit_wait_ms: int = 600_000, device=None):
        super().__init__(torch, budget_bytes, device)
        from . import _lib as L
        from .fft import check

        self.L = L
        self.check = check
        self.max_batch = max_batch
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(streams)]
        self.slot_event = [None] * streams
        self.next = 0
        self.plans = {}
        # The first plans start the run-time compilation of every length's
        # kernels in the background; the plans made after it has finished
        # use them (a plan keeps the kernels it was made with).
        self._make_plans(lengths)
        check(L.lib().sipFftJitWait(jit_wait_ms), "run-time kernels")
        self._destroy_plans()
        self._make_plans(lengths)
        self._first_launches()
        self.prepare_signals(lengths)
        self.launches = 0

    def _first_launches(self) -> None:
        """One row through every plan: CUDA loads a kernel's module on its
        first launch (lazy loading), which would otherwise land on the first
        request of each length.  The rows come from the start of the arena
        (its contents are not used)."""
        s = self.streams[0]
        row = 8 * max(n for _, n in self.plans)
        for h in self.plans.values():
            self.check(h.set_stream(s), "stream")
            self.check(h.exec_rows(1, self.base, self.base + row, self.base + 2 * row), "first launch")
        s.synchronize()

    def _make_plans(self, lengths):
        from .fft import FftHandle

        L, check = self.L, self.check
        for n in lengths:
            for kind in (KIND_PULSE, KIND_FFT):
                h = FftHandle()
                if kind == KIND_PULSE:
                    check(h.make_plan_pulse_1d(n, self.max_batch, self.filter(n).data_ptr(),
                                               L.SIP_FFT_PULSE_CONJ_FILTER), "pulse plan")
                else:
                    check(h.make_plan_1d(n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, self.max_batch), "fft plan")
                check(h.workspace_size()[0], "workspace size")
                self.plans[(kind, n)] = h

    def _destroy_plans(self):
        for h in self.plans.values():
            h.destroy()
        self.plans.clear()

    def _free_slot(self) -> int:
        for k in range(len(self.streams)):
            i = (self.next + k) % len(self.streams)
            ev = self.slot_event[i]
            if ev is None or ev.query():
                return i
        return self.next

    def launch(self, group):
        torch = self.torch
        i = self._free_slot()
        self.next = (i + 1) % len(self.streams)
        s = self.streams[i]
        check = self.check
        with torch.cuda.stream(s):
            for r in group:
                self.make_signal(r, self.view(self.regions(r)[0], r.batch * r.n))
        for r in group:
            x, y, ws = self.regions(r)
            h = self.plans[(r.kind, r.n)]
            check(h.set_stream(s), "stream")
            check(h.exec_rows(r.batch, self.base + x, self.base + y, self.base + ws if ws is not None else None),
                  "exec rows")
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        self.slot_event[i] = ev
        self.launches += 1
        return ev

    def close(self) -> None:
        self._destroy_plans()


class PlainExecutor(_GpuBase):
    """The plain per-request FP32 path: forward C2C, multiply, inverse C2C per
    request on one stream, plans in an LRU cache of (N, batch) like sip_pta."""

    def __init__(self, torch, budget_bytes: int, cache_size: int = 10, device=None):
        super().__init__(torch, budget_bytes, device)
        from . import _lib as L
        from .fft import check

        self.L = L
        self.check = check
        self.streams = [torch.cuda.Stream(device=self.dev)]
        self.cache = collections.OrderedDict()
        self.cache_size = cache_size
        self.hits = 0
        self.misses = 0

    def plans(self, r: Request):
        from .fft import FftHandle

        key = (r.n, r.batch)
        if key in self.cache:
            self.cache.move_to_end(key)
            self.hits += 1
            return self.cache[key]
        self.misses += 1
        L, check = self.L, self.check
        fwd, inv = FftHandle(), FftHandle()
        check(fwd.make_plan_1d(r.n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_FORWARD, r.batch), "plan fwd")
        check(inv.make_plan_1d(r.n, L.ASCEND_FFT_C2C, L.ASCEND_FFT_INVERSE, r.batch), "plan inv")
        for h in (fwd, inv):
            check(h.set_stream(self.streams[0]), "stream")
            check(h.workspace_size()[0], "workspace size")
        self.cache[key] = (fwd, inv)
        if len(self.cache) > self.cache_size:
            _, (f, i) = self.cache.popitem(last=False)
            f.destroy()
            i.destroy()
        return fwd, inv

    def launch(self, group):
        torch = self.torch
        s = self.streams[0]
        check = self.check
        for r in group:
            x, y, ws = self.regions(r)
            fwd, inv = self.plans(r)
            with torch.cuda.stream(s):
                self.make_signal(r, self.view(x, r.batch * r.n))
            if ws is not None:
                check(fwd.set_workspace_ptr(self.base + ws), "workspace")
                check(inv.set_workspace_ptr(self.base + ws), "workspace")
            check(fwd.exec_raw(self.base + x, self.base + y), "exec fwd")
            if r.kind == KIND_PULSE:
                with torch.cuda.stream(s):
                    yv = self.view(y, r.batch * r.n).view(r.batch, r.n)
                    yv.mul_(self.filter(r.n).conj())
                check(inv.exec_raw(self.base + y, self.base + y), "exec inv")
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        return ev

    def close(self) -> None:
        for f, i in self.cache.values():
            f.destroy()
            i.destroy()
        self.cache.clear()

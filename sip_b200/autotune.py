"""Autotuner of the FFT planner, cached per (type, direction, sizes, batch).

The type fixes the data type (C2C: complex64, R2C: float32 in, C2R:
complex64 in).  Candidates are the planner's default (size-specialized
kernels where compiled) and generic tile kernels over transforms per tile,
elements per thread and radix order (sipFftSetPlanHint).  Each candidate is
planned, run `warmup` times and timed over `reps` executions with CUDA
events on device-resident buffers; the fastest is appended to the tune
cache, the file the planner reads at MakePlan when SIP_FFT_TUNE_CACHE names
it.  Each line is "type direction dims batch P E generic order fused
variant jit" (dims like 64x128), and the last matching line wins.

CLI: python -m sip_b200.autotune --type c2c --n 4096 --batch 256 --cache tune.txt
"""
from __future__ import annotations

import argparse
import itertools
import os
from dataclasses import dataclass

from . import _lib as L

TYPES = {"c2c": L.ASCEND_FFT_C2C, "r2c": L.ASCEND_FFT_R2C, "c2r": L.ASCEND_FFT_C2R}


@dataclass(frozen=True)
class Candidate:
    p: int = 0        # transforms per tile (0: planner default)
    e: int = 0        # elements per thread (0: default)
    generic: int = 0  # 1: generic tile kernels only
    order: int = 0    # radix order (0 descending, 1 ascending)
    fused: int = 0    # real lengths above one tile: 0 default, 1 fuse both, 2 fuse neither
    variant: int = -1  # compiled size-specialized variant (-1: automatic)
    jit: int = 0      # run-time compiled kernels: 0 default, 1 always, 2 never

    def line(self, fft_type: int, direction: int, sizes, batch: int) -> str:
        dims = "x".join(str(int(s)) for s in sizes)
        return (f"{fft_type} {direction} {dims} {batch} {self.p} {self.e} {self.generic} {self.order} "
                f"{self.fused} {self.variant} {self.jit}\n")


def candidates(max_p: int = 16) -> list[Candidate]:
    out = [Candidate(), Candidate(fused=1), Candidate(fused=2)] + [Candidate(variant=v) for v in (0, 1, 2, 3)]
    out += [Candidate(jit=1), Candidate(jit=2)]
    ps = [0] + [p for p in (1, 2, 4, 8, 16, 32) if p <= max_p]
    for p, e, order in itertools.product(ps, (16, 32), (0, 1)):
        out.append(Candidate(p, e, 1, order))
    return out


def apply(handle, c: Candidate) -> None:
    from .fft import check

    check(handle.set_hint(L.SIP_FFT_HINT_TILE_TRANSFORMS, c.p), "hint P")
    check(handle.set_hint(L.SIP_FFT_HINT_ELEMS_PER_THREAD, c.e), "hint E")
    check(handle.set_hint(L.SIP_FFT_HINT_GENERIC_ONLY, c.generic), "hint generic")
    check(handle.set_hint(L.SIP_FFT_HINT_RADIX_ORDER, c.order), "hint order")
    check(handle.set_hint(L.SIP_FFT_HINT_REAL_FUSED, c.fused), "hint real fused")
    check(handle.set_hint(L.SIP_FFT_HINT_SK_VARIANT, c.variant), "hint sk variant")
    check(handle.set_hint(L.SIP_FFT_HINT_RUNTIME_COMPILE, c.jit), "hint runtime compile")


def _buffers(torch, fft_type: int, sizes, batch: int, device):
    last = sizes[-1]
    lead = (batch,) + tuple(sizes[:-1])
    if fft_type == L.ASCEND_FFT_C2C:
        x = torch.randn(lead + (last,), dtype=torch.complex64, device=device)
        y = torch.empty_like(x)
    elif fft_type == L.ASCEND_FFT_R2C:
        x = torch.rand(lead + (last,), dtype=torch.float32, device=device)
        y = torch.empty(lead + (last // 2 + 1,), dtype=torch.complex64, device=device)
    else:
        x = torch.randn(lead + (last // 2 + 1,), dtype=torch.complex64, device=device)
        y = torch.empty(lead + (last,), dtype=torch.float32, device=device)
    return x, y


def time_candidate(torch, c: Candidate, fft_type: int, direction: int, sizes, batch: int, x, y,
                   warmup: int = 3, reps: int = 20) -> float:
    """Mean milliseconds per execution, or inf when the candidate does not plan."""
    from .fft import FftHandle, check

    h = FftHandle()
    try:
        apply(h, c)
        if len(sizes) == 1:
            rc = h.make_plan_1d(sizes[0], fft_type, direction, batch)
        elif len(sizes) == 2:
            rc = h.make_plan_2d(sizes[0], sizes[1], fft_type, direction, batch)
        else:
            rc = h.make_plan_3d(sizes[0], sizes[1], sizes[2], fft_type, direction, batch)
        if rc != L.ACL_SUCCESS:
            return float("inf")
        h.bind_workspace(x.device)
        s = torch.cuda.Stream(device=x.device)
        check(h.set_stream(s), "stream")
        torch.cuda.synchronize(x.device)  # inputs were filled on the default stream
        for _ in range(warmup):
            check(h.exec_raw(x.data_ptr(), y.data_ptr()), "exec")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            check(h.exec_raw(x.data_ptr(), y.data_ptr()), "exec")
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        h.destroy()


def tune(fft_type: int, direction: int, sizes, batch: int, cache_path: str | None = None, reps: int = 20,
         cands=None, timer=None) -> dict:
    """Times every candidate; appends the fastest to `cache_path` (when given)
    and returns {"best": Candidate, "ms": best time, "times": {Candidate: ms}}.
    `timer(candidate) -> ms` replaces the GPU timing (tests)."""
    cands = cands if cands is not None else candidates()
    times = {}
    if timer is None:
        import torch

        x, y = _buffers(torch, fft_type, list(sizes), batch, torch.device("cuda"))
        for c in cands:
            times[c] = time_candidate(torch, c, fft_type, direction, list(sizes), batch, x, y, reps=reps)
    else:
        for c in cands:
            times[c] = timer(c)
    best = min(times, key=times.get)
    if times[best] == float("inf"):
        raise RuntimeError("no candidate planned")
    if cache_path:
        with open(cache_path, "a") as f:
            f.write(best.line(fft_type, direction, sizes, batch))
    return {"best": best, "ms": times[best], "times": times}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--type", choices=sorted(TYPES), default="c2c")
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--n", type=int, nargs="+", required=True, help="transform sizes (1-3)")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--cache", default=os.environ.get("SIP_FFT_TUNE_CACHE", "sip_fft_tune.txt"))
    a = ap.parse_args()
    d = L.ASCEND_FFT_INVERSE if a.inverse else L.ASCEND_FFT_FORWARD
    r = tune(TYPES[a.type], d, a.n, a.batch, a.cache, a.reps)
    default = r["times"][Candidate()]
    print(f"best {r['best']} {r['ms']:.4f} ms (planner default {default:.4f} ms) -> {a.cache}")


if __name__ == "__main__":
    main()

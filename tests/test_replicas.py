"""Multi-process replica path on CPU (gloo, world_size 2).

Rows are independent, so bench.py --gpus N runs N replicas of the workload
with no data-path collective: a barrier, and a MAX over ranks of each rank's
measured time.  Here two gloo ranks each run the same seeded transform
through the CPU harness, check it against the FP64 oracle, agree on the
result bit for bit, and reduce a per-rank time with the helper bench.py uses.
"""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, outdir: str) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    from sip_b200.replicas import max_over_ranks, rank_env, reports
    from tests.fftcase import emu_run, random_input
    from tests.native.build_emu import load

    w, r, local = rank_env()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    emu = load()
    x = random_input(O.R2C, [1000], 4, seed=20261029 + 1000)      # same workload on every replica
    rc, out, _ = emu_run(emu, O.R2C, O.FORWARD, [1000], 4, x)
    err = O.rel_l2(out, O.fp64(O.R2C, O.FORWARD, x, [1000]))
    gathered = [None] * w
    dist.all_gather_object(gathered, out.tobytes())
    dist.barrier()
    ms = max_over_ranks(1.0 + rank, dist, "cpu")                  # rank-dependent "time"
    dist.barrier()
    res = {"rank": r, "local": local, "rc": rc, "err": err, "same": all(g == gathered[0] for g in gathered),
           "max_ms": ms, "reports": reports(r)}
    Path(outdir, f"rank{r}.json").write_text(json.dumps(res))
    dist.destroy_process_group()


def test_two_gloo_replicas(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, d in enumerate(res):
        assert d["rank"] == r and d["local"] == r and d["rc"] == 0
        assert d["err"] <= 1e-6
        assert d["same"]
        assert d["max_ms"] == pytest.approx(float(world))          # the slowest rank's time
        assert d["reports"] == (r == 0)


def test_single_process_defaults(monkeypatch):
    from sip_b200.replicas import max_over_ranks, rank_env

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert rank_env() == (1, 0, 0)
    assert max_over_ranks(3.5) == 3.5
    assert np.isfinite(max_over_ranks(0.0))

"""Batched work-queue execution (sipFftBatch*) on the GPU.

Pass k of every plan added to a batch runs in one persistent launch
(sip_b200/csrc/queue.cu).  Each result must be the same whether its plan
runs alone or in a mix of lengths, directions and types, and must match the
plain per-plan execution and the FP64 oracle.
"""
import numpy as np
import pytest

from oracle import oracle as O
from sip_b200 import _lib as L
from tests.fftcase import settle, make_plan, random_input, shapes

pytestmark = pytest.mark.gpu

# (type, direction, sizes, batch)
MIX = [
    (O.C2C, O.FORWARD, [1000], 3),
    (O.C2C, O.INVERSE, [4096], 2),
    (O.R2C, O.FORWARD, [1000], 4),
    (O.C2R, O.INVERSE, [2048], 2),
    (O.R2C, O.FORWARD, [2187], 2),
    (O.C2R, O.INVERSE, [243], 3),
    (O.C2C, O.FORWARD, [65536], 1),
    (O.C2C, O.INVERSE, [64, 128], 2),
    (O.R2C, O.FORWARD, [64, 256], 2),
]


class Job:
    def __init__(self, torch, case, seed):
        from sip_b200.fft import FftHandle, check

        self.case = case
        op, d, sizes, b = case
        self.x = random_input(op, sizes, b, seed)
        _, _, oshape, odt = shapes(op, sizes, b)
        dev = torch.device("cuda")
        self.xt = torch.from_numpy(np.ascontiguousarray(self.x)).to(dev)
        self.yt = torch.zeros(oshape, dtype=torch.complex64 if odt == np.complex64 else torch.float32, device=dev)
        self.h = FftHandle()
        check(self.h.set_hint(L.SIP_FFT_HINT_GENERIC_ONLY, 1), "hint")
        check(make_plan(self.h, op, d, list(sizes), b), "plan")
        self.h.bind_workspace()

    def result(self):
        return self.yt.cpu().numpy()

    def reset(self):
        self.yt.zero_()


def run_batch(torch, jobs, stream, use_graphs=True):
    from sip_b200.fft import Batch, check

    with Batch(use_graphs) as bt:
        for j in jobs:
            check(bt.add(j.h, j.xt.data_ptr(), j.yt.data_ptr()), "batch add")
        settle()
        check(bt.execute(stream), "batch exec")
        stream.synchronize()
        assert bt.take_status() == 0


@pytest.fixture()
def jobs(cuda):
    js = [Job(cuda, c, 100 + i) for i, c in enumerate(MIX)]
    yield js
    for j in js:
        j.h.destroy()


def oracle_check(job, out):
    # the library's accuracy bar, as for the plain exec
    op, d, sizes, b = job.case
    want = O.fp64(op, d, job.x, sizes)
    assert O.rel_l2(out, want) <= 1e-6, job.case


def test_mix_equals_alone_and_plain(cuda, jobs):
    from sip_b200.fft import check

    s = cuda.cuda.Stream()
    run_batch(cuda, jobs, s)
    mixed = [j.result() for j in jobs]
    for j, m in zip(jobs, mixed):
        oracle_check(j, m)
        j.reset()
        run_batch(cuda, [j], s)
        alone = j.result()
        np.testing.assert_array_equal(alone, m, err_msg=str(j.case))  # same kernel, same bits
        j.reset()
        check(j.h.set_stream(s), "stream")
        settle()
        check(j.h.exec_raw(j.xt.data_ptr(), j.yt.data_ptr()), "exec")
        s.synchronize()
        plain = j.result()
        scale = np.abs(plain).max()
        assert np.abs(plain - m).max() <= 1e-6 * scale, j.case


def test_graph_replay_with_new_operands(cuda, jobs):
    """Same wave structure twice (graph replay), different buffers: both right."""
    s = cuda.cuda.Stream()
    run_batch(cuda, jobs[:4], s)
    first = [j.result() for j in jobs[:4]]
    from sip_b200.fft import Batch, check

    with Batch(True) as bt:
        for rep in range(3):
            bt.clear()
            for j in jobs[:4]:
                j.reset()
                check(bt.add(j.h, j.xt.data_ptr(), j.yt.data_ptr()), "add")
            settle()
            check(bt.execute(s), "exec")
            s.synchronize()
            for j, f in zip(jobs[:4], first):
                np.testing.assert_array_equal(j.result(), f)


def test_eager_matches_graph(cuda, jobs):
    s = cuda.cuda.Stream()
    run_batch(cuda, jobs, s, use_graphs=True)
    g = [j.result() for j in jobs]
    for j in jobs:
        j.reset()
    run_batch(cuda, jobs, s, use_graphs=False)
    for j, r in zip(jobs, g):
        np.testing.assert_array_equal(j.result(), r)


def test_gate_timeout_sets_status(cuda, jobs):
    """A gate flag that nothing sets: the launch gives up after its poll
    limit, flags the status word and leaves the outputs untouched."""
    from sip_b200.fft import Batch, check

    s = cuda.cuda.Stream()
    flag = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    j = jobs[0]
    with Batch(False) as bt:
        check(bt.set_gate(flag.data_ptr(), 2000), "gate")
        check(bt.add(j.h, j.xt.data_ptr(), j.yt.data_ptr()), "add")
        settle()
        check(bt.execute(s), "exec")
        s.synchronize()
        assert bt.take_status() == L.SIP_FFT_BATCH_GATE_TIMEOUT
        assert not j.result().any()
        flag.fill_(1)
        settle()
        check(bt.execute(s), "exec")
        s.synchronize()
        assert bt.take_status() == 0
    oracle_check(j, j.result())


def test_rejects_specialized_plan(cuda):
    from sip_b200.fft import Batch, FftHandle, check

    h = FftHandle()
    check(h.make_plan_1d(4096, O.C2C, O.FORWARD, 64), "plan")
    x = cuda.zeros(64 * 4096, dtype=cuda.complex64, device="cuda")
    with Batch() as bt:
        assert bt.add(h, x.data_ptr(), x.data_ptr()) == L.ACL_ERROR_API_NOT_SUPPORT
    h.destroy()


def test_graph_replay_with_changing_item_counts(cuda, jobs):
    """Replays of one captured graph (same wave count) with different numbers
    of items per wave: the item offsets travel in the uploaded headers."""
    from sip_b200.fft import Batch, check

    s = cuda.cuda.Stream()
    run_batch(cuda, jobs, s)
    want = {id(j): j.result() for j in jobs}
    two_pass = [j for j in jobs if len(j.h.describe()["steps"]) == 2]
    one_pass = [j for j in jobs if len(j.h.describe()["steps"]) == 1]
    assert two_pass and len(one_pass) >= 3
    with Batch(True) as bt:
        for k in range(1, len(one_pass) + 1):
            bt.clear()
            sel = one_pass[:k] + two_pass          # wave 0 grows, wave 1 stays
            for j in sel:
                j.reset()
                check(bt.add(j.h, j.xt.data_ptr(), j.yt.data_ptr()), "add")
            settle()
            check(bt.execute(s), "exec")
            s.synchronize()
            assert bt.take_status() == 0
            for j in sel:
                np.testing.assert_array_equal(j.result(), want[id(j)])

"""Serving loop host logic on CPU, with a fake prover context: admission by
the memory budget, head-of-line order, per-request failure reporting."""
import threading
import time

import numpy as np

from loom_b200 import serve as S


class FakeContext:
    running = 0
    peak = 0
    lock = threading.Lock()

    def __init__(self, device):
        self.order = []

    def set_batched(self, b):
        pass

    def mem_info(self):
        return 1 << 40, 1 << 40

    def prove(self, words, witness, q):
        with FakeContext.lock:
            FakeContext.running += 1
            FakeContext.peak = max(FakeContext.peak, FakeContext.running)
        time.sleep(0.01 * q)
        with FakeContext.lock:
            FakeContext.running -= 1
        if q == 7:
            raise RuntimeError("injected failure")
        return bytes([q]) * 4

    def close(self):
        pass


def reqs(sizes, qs):
    return [S.Request(i, np.zeros(1, np.uint32), [], q, rows) for i, (rows, q) in enumerate(zip(sizes, qs))]


def test_budget_limits_concurrency():
    FakeContext.peak = 0
    rows = 1 << 16
    budget = 2 * S.device_bytes_estimate(rows) + 1  # room for two at a time
    rs = reqs([rows] * 8, [2] * 8)
    res = S.serve(rs, [0.0] * 8, streams=4, hbm_budget=budget, context_factory=FakeContext)
    assert res["errors"] == 0 and len(res["finished"]) == 8
    assert res["peak_budget_in_use"] <= budget
    assert FakeContext.peak <= 2


def test_oversized_request_runs_alone_and_in_order():
    rows_small, rows_big = 1 << 10, 1 << 30
    rs = reqs([rows_small, rows_big, rows_small], [1, 1, 1])
    res = S.serve(rs, [0.0, 0.001, 0.002], streams=3, hbm_budget=S.device_bytes_estimate(rows_small) * 4,
                  context_factory=FakeContext)
    assert res["errors"] == 0
    starts = {r.rid: r.start for r in res["finished"]}
    assert starts[0] <= starts[1] <= starts[2]  # head of line: no overtaking


def test_failure_is_reported_per_request():
    rs = reqs([1024] * 4, [1, 7, 1, 1])
    res = S.serve(rs, [0.0] * 4, streams=2, hbm_budget=1 << 40, context_factory=FakeContext)
    assert res["errors"] == 1
    bad = [r for r in res["finished"] if r.error]
    assert bad[0].rid == 1 and "injected failure" in bad[0].error
    assert all(r.proof == bytes([1]) * 4 for r in res["finished"] if not r.error)


def test_poisson_arrivals_are_seeded_and_increasing():
    a = S.poisson_arrivals(100, 50.0, 3)
    assert np.all(np.diff(a) > 0) and np.array_equal(a, S.poisson_arrivals(100, 50.0, 3))
    assert 1.0 < a[-1] < 4.0


def test_close_waits_for_requests_in_flight():
    """A context is destroyed only after its running prove returns, and a
    closed server admits nothing more."""
    events = []

    class SlowContext(FakeContext):
        def prove(self, words, witness, q):
            time.sleep(0.2)
            events.append(("proved", id(self)))
            return b"ok"

        def close(self):
            events.append(("closed", id(self)))

    srv = S.Server(streams=2, hbm_budget=1 << 40, context_factory=SlowContext)
    rs = reqs([1024] * 3, [1, 1, 1])
    for r in rs:
        srv.submit(r)
    srv.close()
    assert sorted(e for e, _ in events) == ["closed", "closed", "proved", "proved"]
    for ctx_id in {i for _, i in events}:
        mine = [e for e, i in events if i == ctx_id]
        assert mine == ["proved", "closed"]
    assert len(srv.finished) == 2 and srv.queue == [rs[2]]  # the third was never admitted

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


class DeviceModel:
    """A fake device for the admission tests: bytes in use, and a total."""

    def __init__(self, total):
        self.total, self.used = total, 0
        self.lock = threading.Lock()

    def available(self):
        with self.lock:
            return self.total - self.used


def test_waits_for_live_memory_and_learns_the_measured_need():
    """Admission reads the device's allocatable bytes when it decides: a
    request whose measured need does not fit next to a running prove waits
    for that prove to free its memory, then starts; the need it learns is the
    peak each prove took (the contexts' high-water marks)."""
    dev = DeviceModel(total=1000)
    starts, ends = {}, {}

    class MemContext(FakeContext):
        def __init__(self, device):
            super().__init__(device)
            self.held = self.peak_mark = 0

        def mem_usage(self, reset_peak=False):
            if reset_peak:
                self.peak_mark = self.held
            return self.held, self.peak_mark

        def device_available(self):
            return dev.available()

        def prove(self, words, witness, q):
            rid = int(words[0])
            starts[rid] = time.perf_counter()
            with dev.lock:
                dev.used += 600  # each prove takes 600 of the 1000 bytes at its peak
                self.held += 600
                self.peak_mark = max(self.peak_mark, self.held)
            time.sleep(0.05)
            with dev.lock:
                dev.used -= 600
                self.held -= 600
            ends[rid] = time.perf_counter()
            return b"p"

    rs = [S.Request(i, np.array([i], np.uint32), [], 1, 16) for i in range(3)]
    srv = S.Server(streams=3, hbm_budget=None, context_factory=MemContext, margin=0)
    srv.measured[rs[0].shape()] = 600  # as a warm-up would have measured
    srv.measured[rs[1].shape()] = 600
    srv.measured[rs[2].shape()] = 600
    for r in rs:
        srv.submit(r)
    srv.wait(3, timeout=10)
    srv.close()
    # three free streams, yet the memory admits one prove at a time
    assert starts[1] >= ends[0] and starts[2] >= ends[1]
    assert srv.waits_for_memory >= 2
    assert all(r.peak_bytes == 600 for r in srv.finished)
    # a shape seen for the first time starts from the per-row prior, then
    # runs on what it measured
    srv2 = S.Server(streams=1, context_factory=MemContext, margin=0)
    r = S.Request(9, np.array([9], np.uint32), [], 1, 1 << 12)
    assert srv2.need(r) == S.device_bytes_estimate(1 << 12)
    srv2.submit(r)
    srv2.wait(1, timeout=10)
    srv2.close()
    assert srv2.need(r) == 600

"""Serving loop: proving requests of mixed sizes arriving over time.

Requests wait in arrival order.  A request starts as soon as a stream slot is
free and its device memory fits (continuous batching: no request waits for a
batch to drain; proofs of different requests overlap on the GPU, one CUDA
stream each).  Its memory need is the peak the library measured for the same
request shape before (each context's high-water mark around a prove,
lg_ctx_mem_usage), or a per-row estimate for a shape not seen yet; it fits
when the device's allocatable bytes at admission time (lg_device_mem_info:
free memory plus the memory pool's unused reserve) cover it next to what the
running requests have still to allocate of theirs.  An optional static budget
caps the sum of the running requests' needs as well.  The witness of a
running request and all its LDEs and trees stay on the device until its
proof is read back.  Every proof is a pure function of its request, so a
request's bytes are the same alone and in the mix.

Latency = completion time - arrival time.  Reports p50/p99 and proofs/s.
"""
from __future__ import annotations

import heapq
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import field as F, plonk
from ._lib import Context


@dataclass
class Request:
    rid: int
    words: np.ndarray
    witness: List[np.ndarray]     # Montgomery columns, descriptor order
    num_queries: int
    rows: int                     # total trace rows (sum over modules)
    arrival: float = 0.0
    start: float = 0.0
    done: float = 0.0
    proof: Optional[bytes] = None
    error: Optional[str] = None
    peak_bytes: int = 0           # device bytes the prove took at its peak (measured)

    def shape(self):
        """Requests of one shape (program and query count) need the same memory."""
        return (hash(np.ascontiguousarray(self.words).tobytes()), self.num_queries)


def device_bytes_estimate(rows: int) -> int:
    """Prior for a request shape not measured yet: peak device bytes of one
    prove of plonk-like modules totalling `rows` rows (LDEs and coefficients
    of the committed columns at blowup 4, quotient scratch, DEEP codewords and
    trees), 2.2 KiB per row with headroom."""
    return int(2304 * rows) + (64 << 20)


def make_request(rid: int, log_rows: int, instances: int, num_queries: int, seed: int) -> Request:
    compiled, wit = plonk.build(instances, 1 << log_rows, seed=seed)
    mont = [np.ascontiguousarray(F.to_mont(w)) for w in wit]
    return Request(rid, compiled.words, mont, num_queries, instances << log_rows)


class Server:
    """`hbm_budget`: a static cap on the running requests' summed needs (None:
    none).  `mem_probe`: callable giving the device bytes allocatable now
    (default: the contexts' device_available(), when they have it).
    `margin`: bytes kept free beyond every admission."""

    def __init__(self, streams: int = 4, device: int = 0, hbm_budget: Optional[int] = None,
                 batched: bool = True, context_factory: Optional[Callable[[int], object]] = None,
                 tuning: Optional[dict] = None, mem_probe: Optional[Callable[[], int]] = None,
                 margin: int = 256 << 20):
        make = context_factory or Context
        self.contexts = [make(device) for _ in range(streams)]
        for c in self.contexts:
            c.set_batched(batched)
            if tuning:
                c.apply_tuning(tuning)
        c0 = self.contexts[0]
        self.mem_probe = mem_probe or (c0.device_available if hasattr(c0, "device_available") else None)
        self.margin = margin if self.mem_probe else 0
        self.budget = hbm_budget if hbm_budget is not None else float("inf")
        self.measured: Dict[tuple, int] = {}  # request shape -> measured peak bytes
        self.flight: Dict[int, tuple] = {}     # rid -> (context, need, device bytes it held at start)
        self.waits_for_memory = 0              # admissions deferred for live device memory
        self.in_use = 0
        self.cv = threading.Condition()
        self.queue: List[Request] = []     # arrival order
        self.idle = list(self.contexts)
        self.finished: List[Request] = []
        self.peak_in_use = 0
        self.running = 0                   # requests in flight
        self.closed = False
        self.t0 = time.perf_counter()

    def warm(self, requests: Sequence[Request]):
        """Runs each distinct request once on every context, so twiddle tables,
        pinned staging and the device memory pool exist before timing; the
        peaks measured on the way are the admission's needs for those shapes."""
        for ctx in self.contexts:
            for r in requests:
                base = ctx.mem_usage(reset_peak=True)[0] if hasattr(ctx, "mem_usage") else None
                ctx.prove(r.words, r.witness, r.num_queries)
                if base is not None:
                    k = r.shape()
                    self.measured[k] = max(self.measured.get(k, 0), ctx.mem_usage()[1] - base)

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def need(self, r: Request) -> int:
        return self.measured.get(r.shape(), device_bytes_estimate(r.rows))

    @staticmethod
    def _held(ctx) -> Optional[int]:
        return ctx.mem_usage()[0] if hasattr(ctx, "mem_usage") else None

    def _outstanding(self) -> int:
        """What the running requests have still to allocate of their needs."""
        tot = 0
        for ctx, need, base in self.flight.values():
            held = self._held(ctx)
            grown = 0 if held is None or base is None else max(0, held - base)
            tot += max(0, need - grown)
        return tot

    def _admit(self) -> List[tuple]:
        """Head-of-line admission: the oldest request starts when a slot and
        its memory are free (no reordering, so no request starves); with
        nothing running it starts whatever its need."""
        started = []
        while self.queue and self.idle and not self.closed:
            r = self.queue[0]
            need = self.need(r)
            if self.running > 0:
                if self.in_use + need > self.budget:
                    break
                if self.mem_probe is not None and need + self._outstanding() + self.margin > self.mem_probe():
                    self.waits_for_memory += 1
                    break
            self.queue.pop(0)
            self.running += 1
            self.in_use += need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            ctx = self.idle.pop()
            self.flight[r.rid] = (ctx, need, self._held(ctx))
            started.append((r, ctx, need))
        return started

    def _run(self, r: Request, ctx: Context, need: int):
        r.start = self.now()
        base = None
        if hasattr(ctx, "mem_usage"):
            base = ctx.mem_usage(reset_peak=True)[0]
        try:
            r.proof = ctx.prove(r.words, r.witness, r.num_queries)
        except Exception as e:  # reported per request
            r.error = str(e)
        if base is not None:
            r.peak_bytes = max(0, ctx.mem_usage()[1] - base)
        r.done = self.now()
        with self.cv:
            if r.peak_bytes and r.error is None:
                k = r.shape()
                self.measured[k] = max(self.measured.get(k, 0), r.peak_bytes)
            self.flight.pop(r.rid, None)
            self.running -= 1
            self.in_use -= need
            self.idle.append(ctx)
            self.finished.append(r)
            for item in self._admit():
                threading.Thread(target=self._run, args=item, daemon=True).start()
            self.cv.notify_all()

    def submit(self, r: Request):
        with self.cv:
            r.arrival = self.now()
            self.queue.append(r)
            for item in self._admit():
                threading.Thread(target=self._run, args=item, daemon=True).start()

    def wait(self, n: int, timeout: float = 3600.0):
        with self.cv:
            self.cv.wait_for(lambda: len(self.finished) >= n, timeout=timeout)

    def close(self, timeout: Optional[float] = None):
        """Admits nothing more, waits for the requests in flight (a context
        must not be destroyed under a running prove), then destroys the
        contexts.  A context still proving when `timeout` runs out is left
        to the process exit rather than freed under its prove."""
        with self.cv:
            self.closed = True
            self.cv.wait_for(lambda: self.running == 0, timeout=timeout)
            idle = list(self.idle)
            self.idle = []
        for c in idle:
            c.close()


def poisson_arrivals(n: int, rate_per_s: float, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))


def serve(requests: Sequence[Request], arrivals: Sequence[float], streams: int = 4, device: int = 0,
          hbm_budget: Optional[int] = None, batched: bool = True,
          context_factory: Optional[Callable[[int], object]] = None,
          warm: Sequence[Request] = (), tuning: Optional[dict] = None,
          mem_probe: Optional[Callable[[], int]] = None) -> Dict:
    """Replays `requests` at the given arrival offsets (seconds); returns
    latency percentiles, throughput and the finished requests.  `warm`
    requests run once per context before the clock starts (and give the
    admission its measured needs)."""
    srv = Server(streams, device, hbm_budget, batched, context_factory, tuning, mem_probe)
    try:
        srv.warm(warm)
        srv.t0 = time.perf_counter()
        t_start = srv.now()
        for r, at in zip(requests, arrivals):
            delay = t_start + at - srv.now()
            if delay > 0:
                time.sleep(delay)
            srv.submit(r)
        srv.wait(len(requests))
        t_end = srv.now()
        lat = np.array([(r.done - r.arrival) * 1e3 for r in srv.finished])
        return {
            "requests": len(requests),
            "streams": streams,
            "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()),
            "proofs_per_s": len(requests) / (t_end - t_start),
            "errors": sum(r.error is not None for r in srv.finished),
            "first_error": next((r.error for r in srv.finished if r.error), None),
            "peak_budget_in_use": srv.peak_in_use,
            "budget": srv.budget if srv.budget != float("inf") else None,
            "measured_need_bytes": sorted(srv.measured.values()),
            "admissions_deferred_for_memory": srv.waits_for_memory,
            "finished": srv.finished,
        }
    finally:
        srv.close()

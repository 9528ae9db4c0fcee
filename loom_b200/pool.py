"""Concurrent proving on one GPU: a pool of contexts, one CUDA stream and one
host thread each.  While one proof waits on the transcript (roots read back,
challenges hashed on the host), the others keep the GPU busy; the library
releases the Python GIL during each call.

A request is (program words, witness columns, num_queries); results are the
canonical proof bytes, identical to a proof made alone (every proof owns its
transcript and buffers; only the device is shared).
"""
from __future__ import annotations

import queue
import threading
from concurrent.futures import Future
from typing import List, Optional, Sequence

from ._lib import Context


class ProverPool:
    def __init__(self, streams: int, device: int = 0, tuning: Optional[dict] = None):
        self.contexts: List[Context] = [Context(device, tuning) for _ in range(streams)]
        self._q: "queue.Queue[Optional[tuple]]" = queue.Queue()
        self._threads = [threading.Thread(target=self._worker, args=(c,), daemon=True) for c in self.contexts]
        for t in self._threads:
            t.start()

    def _worker(self, ctx: Context):
        while True:
            item = self._q.get()
            if item is None:
                return
            fut, words, witness, q, on_device = item
            if not fut.set_running_or_notify_cancel():
                continue
            try:
                fut.set_result(ctx.prove(words, witness, q, on_device=on_device))
            except BaseException as e:  # surfaced to the caller through the future
                fut.set_exception(e)

    def submit(self, words, witness: Sequence, num_queries: int, on_device: bool = False) -> Future:
        fut: Future = Future()
        self._q.put((fut, words, witness, num_queries, on_device))
        return fut

    def close(self):
        for _ in self._threads:
            self._q.put(None)
        for t in self._threads:
            t.join()
        for c in self.contexts:
            c.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

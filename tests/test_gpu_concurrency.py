"""Concurrent proofs of different sizes on one GPU (one context per thread):
each equals the proof made alone."""
import threading

import pytest

from loom_b200 import Context, field as F, plonk

pytestmark = pytest.mark.gpu


def test_concurrent_contexts_mixed_sizes():
    shapes = [(12, 2), (9, 3), (14, 1), (10, 4), (12, 1), (8, 2)]
    jobs = []
    for i, (lg, inst) in enumerate(shapes):
        comp, wit = plonk.build(inst, 1 << lg, seed=900 + i)
        jobs.append((comp.words, [F.to_mont(w) for w in wit]))
    c0 = Context(0)
    alone = [c0.prove(w, m, 5) for (w, m) in jobs]
    c0.close()
    ctxs = [Context(0) for _ in range(3)]
    out = {}
    errs = []

    def worker(t):
        try:
            for rep in range(3):
                for i in range(t, len(jobs), 3):
                    out[(rep, i)] = ctxs[t].prove(jobs[i][0], jobs[i][1], 5)
        except Exception as e:
            errs.append(e)

    th = [threading.Thread(target=worker, args=(t,)) for t in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in ctxs:
        c.close()
    assert not errs, errs
    for (rep, i), pb in out.items():
        assert pb == alone[i], (rep, i)

"""Serving on the GPU: every proof is the same alone and in the mix of
concurrently running requests of different sizes (exact equality)."""
import numpy as np
import pytest

import oracle
from loom_b200 import Context, serve as S

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix():
    rng = np.random.Generator(np.random.PCG64(42))
    shapes = [(int(rng.integers(8, 12)), int(rng.integers(1, 4)), int(rng.integers(2, 9))) for _ in range(12)]
    reqs = [S.make_request(i, lg, inst, q, seed=100 + i) for i, (lg, inst, q) in enumerate(shapes)]
    ctx = Context(0)
    alone = [ctx.prove(r.words, r.witness, r.num_queries) for r in reqs]
    ctx.close()
    res = S.serve(reqs, S.poisson_arrivals(len(reqs), 400.0, 7), streams=3)
    assert res["errors"] == 0 and len(res["finished"]) == len(reqs)
    for r in res["finished"]:
        assert r.proof == alone[r.rid], f"request {r.rid} differs in the mix"
    for r in reqs[:2]:
        assert alone[r.rid] == oracle.prove(r.words, r.witness, r.num_queries)

"""The headline workload at full size against the oracle: 40 plonk-like
modules of 2^14 rows (copy constraint, grand product), Poseidon2, 200
queries.  The oracle takes about a minute on the host cores; the proof must
be the same bytes, and both the oracle's verifier and the library's must
accept it."""
import numpy as np
import pytest

import oracle
from loom_b200 import field as F, plonk, proof

pytestmark = pytest.mark.gpu


def test_forty_modules_of_2e14_equal_oracle(ctx):
    compiled, wit = plonk.build(40, 1 << 14, seed=0x10AD)
    mont = [np.ascontiguousarray(F.to_mont(w)) for w in wit]
    got = ctx.prove(compiled.words, mont, 200)
    want = oracle.prove(compiled.words, mont, 200)
    assert len(got) == len(want)
    assert got == want
    p = proof.decode(got)
    assert all(v == p.final_poly[0] for v in p.final_poly)
    oracle.verify(compiled.words, got, 200)
    ctx.verify(compiled.words, got, 200)

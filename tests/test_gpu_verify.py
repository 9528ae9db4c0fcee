"""The library's verifier (lg_verify: host transcript, AIR and FRI checks;
Merkle openings and DEEP bridge on the GPU) against the oracle's verifier:
the same proofs are accepted, false statements and tampered proofs rejected
by both."""
import numpy as np
import pytest

import oracle
from loom_b200 import LoomError, field as F, plonk

pytestmark = pytest.mark.gpu


def _both_accept(ctx, words, pb, q, **kw):
    oracle_kw = dict(kw)
    if kw.get("setup_root") is not None:
        oracle_kw["setup_root"] = F.from_mont(kw["setup_root"])
    oracle.verify(words, pb, q, **oracle_kw)
    ctx.verify(words, pb, q, **kw)


def _rejects(ctx, words, pb, q, **kw):
    with pytest.raises(LoomError) as e:
        ctx.verify(words, pb, q, **kw)
    assert e.value.code == 1 and "rejected" in str(e.value)
    return str(e.value)


def test_accepts_plonk_and_rejects_bit_flips(ctx):
    compiled, wit = plonk.build(3, 1 << 10, seed=41)
    mont = [F.to_mont(w) for w in wit]
    pb = ctx.prove(compiled.words, mont, 32)
    _both_accept(ctx, compiled.words, pb, 32)
    rng = np.random.default_rng(5)
    for _ in range(40):
        i, bit = int(rng.integers(0, len(pb))), int(rng.integers(0, 8))
        b = bytearray(pb)
        b[i] ^= 1 << bit
        with pytest.raises(LoomError):
            ctx.verify(compiled.words, bytes(b), 32)


def test_rejects_false_gate(ctx):
    compiled, wit = plonk.build(2, 1 << 9, seed=43)
    names = [n for (n, _, _) in compiled.witness_columns]
    mont = [F.to_mont(w) for w in wit]
    i = names.index("O_1")
    mont[i] = mont[i].copy()
    mont[i][17] = F.to_mont(np.array([(int(F.from_mont(mont[i][17:18])[0]) + 1) % F.P], dtype=np.uint32))[0]
    pb = ctx.prove(compiled.words, mont, 16)
    assert "AIR relation" in _rejects(ctx, compiled.words, pb, 16)


def test_lookup_bus_ratio_setup(ctx):
    compiled, wit = plonk.build_mixed([9, 6, 10, 7], seed=44)
    pb = ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 24)
    _both_accept(ctx, compiled.words, pb, 24, logup_buses=compiled.logup_buses)
    bus = [compiled.logup_buses[0][0], compiled.logup_buses[1][1]]
    assert "sum to zero" in _rejects(ctx, compiled.words, pb, 24, logup_buses=[bus])

    compiled, wit, ends = plonk.build_with_bus(1 << 8, seed=45, balanced=False)
    pb = ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 12)
    _both_accept(ctx, compiled.words, pb, 12)
    assert "multiply to one" in _rejects(ctx, compiled.words, pb, 12, product_buses=compiled.product_buses)

    compiled, wit = plonk.build_with_tuple_lookup(1 << 8, seed=46)
    pb = ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 12)
    _both_accept(ctx, compiled.words, pb, 12, logup_buses=compiled.logup_buses)

    compiled, wit, setup = plonk.build_with_setup(2, 1 << 8, seed=47)
    root = ctx.setup(compiled.words, [F.to_mont(x) for x in setup])
    pb = ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 12)
    _both_accept(ctx, compiled.words, pb, 12, setup_root=root)
    _rejects(ctx, compiled.words, pb, 12)
    bad = root.copy()
    bad[3] ^= 1
    _rejects(ctx, compiled.words, pb, 12, setup_root=bad)

"""The oracle's verifier (a restatement of verifier/verifier.go and
internal/fri/verify.go) on oracle proofs: valid proofs are accepted, proofs
of false statements and tampered proofs are rejected.  The GPU proofs go
through the same verifier in the `gpu` tests."""
import struct

import numpy as np
import pytest

import oracle
from loom_b200 import field as F, plonk, proof


def _prove(compiled, wit, q):
    return oracle.prove(compiled.words, [F.to_mont(w) for w in wit], q)


@pytest.fixture(scope="module")
def small():
    compiled, wit = plonk.build(2, 1 << 8, seed=11)
    return compiled, wit, _prove(compiled, wit, 12)


@pytest.fixture(scope="module")
def mixed():
    compiled, wit = plonk.build_mixed([6, 5, 7, 4], seed=21)
    return compiled, wit, _prove(compiled, wit, 8)


def test_accepts_plonk_proof(small):
    compiled, _, pb = small
    oracle.verify(compiled.words, pb, 12)


def test_accepts_lookup_proof_with_its_buses(mixed):
    compiled, _, pb = mixed
    assert len(compiled.logup_buses) == 4 and all(len(b) == 2 for b in compiled.logup_buses)
    oracle.verify(compiled.words, pb, 8, compiled.logup_buses)


def test_unbalanced_logup_bus_is_rejected(mixed):
    """Totals of two different lookups do not cancel each other."""
    compiled, _, pb = mixed
    bus = [compiled.logup_buses[0][0], compiled.logup_buses[1][1]]
    with pytest.raises(oracle.VerifyError, match="do not sum to zero"):
        oracle.verify(compiled.words, pb, 8, [bus])


@pytest.mark.parametrize("permuted", [True, False])
def test_running_ratio_product_bus(permuted):
    compiled, wit, end = plonk.build_with_ratio(64, seed=5, permuted=permuted)
    assert compiled.product_buses == [[end]]
    pb = _prove(compiled, wit, 8)
    oracle.verify(compiled.words, pb, 8)  # the constraints hold either way
    if permuted:
        oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)
    else:
        with pytest.raises(oracle.VerifyError, match="do not multiply to one"):
            oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)


@pytest.mark.parametrize("balanced", [True, False])
def test_bus_argument(balanced):
    """arguments.Bus between two modules: the ends of the two running-ratio
    columns multiply to one exactly when the received tuples are the sent
    ones."""
    compiled, wit, ends = plonk.build_with_bus(64, seed=9, balanced=balanced)
    pb = _prove(compiled, wit, 8)
    oracle.verify(compiled.words, pb, 8)  # every constraint holds either way
    if balanced:
        oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)
    else:
        with pytest.raises(oracle.VerifyError, match="do not multiply to one"):
            oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)


def test_false_gate_is_rejected(small):
    compiled, wit, _ = small
    names = [n for (n, _, _) in compiled.witness_columns]
    bad = [w.copy() for w in wit]
    bad[names.index("O_0")][3] = (int(bad[names.index("O_0")][3]) + 1) % F.P
    with pytest.raises(oracle.VerifyError, match="AIR relation"):
        oracle.verify(compiled.words, _prove(compiled, bad, 12), 12)


def test_broken_copy_constraint_is_rejected():
    compiled, wit = plonk.build(1, 1 << 6, seed=13)
    names = [n for (n, _, _) in compiled.witness_columns]
    wit = [w.copy() for w in wit]
    sig = wit[names.index("plonk.S_0_0")]
    sig[[1, 2]] = sig[[2, 1]]
    with pytest.raises(oracle.VerifyError, match="AIR relation"):
        oracle.verify(compiled.words, _prove(compiled, wit, 4), 4)


@pytest.mark.parametrize("case,flips", [("small", 500), ("mixed", 250)])
def test_every_single_bit_flip_is_rejected(small, mixed, case, flips):
    """Random single-bit flips anywhere in the proof (values, digests, paths,
    rows, counts, names) never verify."""
    compiled, _, pb = small if case == "small" else mixed
    q = 12 if case == "small" else 8
    rng = np.random.default_rng(7)
    accepted = []
    for _ in range(flips):
        i, bit = int(rng.integers(0, len(pb))), int(rng.integers(0, 8))
        b = bytearray(pb)
        b[i] ^= 1 << bit
        try:
            oracle.verify(compiled.words, bytes(b), q, compiled.logup_buses)
            accepted.append((i, bit))
        except oracle.VerifyError:
            pass
    assert accepted == []


def test_wrong_query_count_or_program_is_rejected(small, mixed):
    compiled, _, pb = small
    with pytest.raises(oracle.VerifyError):
        oracle.verify(compiled.words, pb, 11)
    with pytest.raises(oracle.VerifyError):
        oracle.verify(mixed[0].words, pb, 12)
    with pytest.raises(oracle.VerifyError, match="truncated"):
        oracle.verify(compiled.words, pb[:-4], 12)


def test_setup_precommit():
    """setup.Setup (setup/setup.go:68-124): selectors, copy permutation and
    identity columns as setup columns go into one precommitted tree whose root
    is the verification key; the proof's commitments leave it out, its claimed
    values and openings come first, and only the right key verifies."""
    compiled, wit, setup = plonk.build_with_setup(2, 64)
    sm = [F.to_mont(x) for x in setup]
    pb = oracle.prove(compiled.words, [F.to_mont(w) for w in wit], 8, sm)
    root = oracle.setup_root(compiled.words, sm)
    oracle.verify(compiled.words, pb, 8, setup_root=root)
    p = proof.decode(pb)
    assert len(p.commitments) == 3 and len(p.claimed_values) == 4
    assert [len(g["base"]) for g in p.claimed_values[0]] == [11, 11]  # 5 selectors, 3 sigma, 3 ID
    assert [len(g["base"]) for g in p.claimed_values[1]] == [3, 3]    # L, R, O only
    with pytest.raises(oracle.VerifyError, match="verification key"):
        oracle.verify(compiled.words, pb, 8)
    bad = root.copy()
    bad[0] ^= 1
    with pytest.raises(oracle.VerifyError):
        oracle.verify(compiled.words, pb, 8, setup_root=bad)
    other = plonk.build_with_setup(2, 64, seed=7)[2]
    assert (oracle.setup_root(compiled.words, [F.to_mont(x) for x in other]) != root).any()


def test_conditional_tuple_lookup():
    """arguments.CLookupUnionTuple: width-2 tuples from two modules with
    selectors (weights 1 and 2) into a table with a selector (values 0, 1, 3)
    and repeated tuples; the proof verifies with its logup bus, and a selected
    source tuple missing from the table is refused by the prover."""
    compiled, wit = plonk.build_with_tuple_lookup(64)
    pb = _prove(compiled, wit, 8)
    oracle.verify(compiled.words, pb, 8, compiled.logup_buses)
    p = proof.decode(pb)
    assert all(v == p.final_poly[0] for v in p.final_poly)
    compiled, wit = plonk.build_with_tuple_lookup(64, present=False)
    with pytest.raises(RuntimeError, match="not in the table"):
        _prove(compiled, wit, 8)


def test_mixed_trace_round_trip_and_tampered_injection_row():
    """verifier_test.go TestVerifyMixedTraceRoundTrip (the fixture of
    prover_test.go TestVanishingRelationsAndLogupBus): a Fibonacci module of 4
    rows (shifted columns, constraints except at the last row) looks up A, B
    and C in a range module of 8 rows, so the trace tree injects the smaller
    group; the proof verifies with its logup buses, and a tampered injection
    row is rejected."""
    from loom_b200.program import Builder, Module, col, lookup
    n = 4
    b = Builder()
    fib = Module("fibonacci", n)
    fib.assert_zero_except_at(col("A", 1) - col("B"), n - 1)
    fib.assert_zero_except_at(col("B", 1) - col("C"), n - 1)
    fib.assert_zero(col("C") - col("A") - col("B"))
    b.add_module(fib)
    b.add_module(Module("range", 2 * n))
    for name in ("A", "B", "C"):
        lookup(b, [(col(name), "fibonacci")], [(col("Lookup"), "range")])
    compiled = b.compile()
    # prover.TraceFibonacci(4, 0, 1) and prover.TraceRange(4) (prover/test_utils.go:58-92)
    trace = {"A": [0, 1, 1, 2], "B": [1, 1, 2, 3], "C": [1, 2, 3, 5], "Lookup": list(range(2 * n))}
    trace.update(b.generated)
    wit = [np.array(trace[name], dtype=np.uint32) for (name, _, _) in compiled.witness_columns]
    pb = _prove(compiled, wit, 8)
    assert len(compiled.logup_buses) == 3
    oracle.verify(compiled.words, pb, 8, compiled.logup_buses)

    p = proof.decode(pb)
    # prover_test.go TestVanishingRelationsAndLogupBus: every logup total is
    # exposed with exactly one entry, and the totals of each bus sum to zero
    for bus_totals in compiled.logup_buses:
        assert all(len(p.exposed[name]) == 1 for name in bus_totals)
        sums = [sum(p.exposed[name][0][2][k] for name in bus_totals) % F.P for k in range(6)]
        assert sums == [0] * 6
    rows = [inj[0] for per in p.point_samplings for wp in per for inj in wp.injections]
    assert rows, "the mixed-size trace tree opens injection rows"
    words = rows[0].base
    at = pb.find(struct.pack(">%dI" % len(words), *words))
    assert at > 0
    bad = bytearray(pb)
    bad[at + 3] ^= 1
    with pytest.raises(oracle.VerifyError):
        oracle.verify(compiled.words, bytes(bad), 8, compiled.logup_buses)

    # a wrong Fibonacci step is caught by the AIR relation
    trace["C"] = [1, 2, 3, 6]
    wit = [np.array(trace[name], dtype=np.uint32) for (name, _, _) in compiled.witness_columns]
    with pytest.raises(oracle.VerifyError, match="AIR relation"):
        oracle.verify(compiled.words, _prove(compiled, wit, 8), 8, compiled.logup_buses)


def _one_module(n):
    from loom_b200.program import Builder, Module
    b = Builder()
    b.add_module(Module("m", n))
    return b


def _witness(b, compiled, trace):
    trace = dict(trace)
    trace.update(b.generated)
    return [np.asarray(trace[name], dtype=np.uint32) for (name, _, _) in compiled.witness_columns]


@pytest.mark.parametrize("bad", [False, True])
def test_bus_within_one_module(bad):
    """bus_test.go TestBusSameModule: sender and receiver in one module share
    one running-ratio column, so the product bus has one end; receiving a
    value that is not sent is rejected."""
    from loom_b200.program import bus, col
    n = 8
    b = _one_module(n)
    ends = bus(b, [col("m.s")], [col("m.r")], [([col("m.x")], "m")], [([col("m.y")], "m")])
    compiled = b.compile()
    assert compiled.product_buses == [ends] and len(ends) == 1
    pad = lambda *v: list(v) + [0] * (n - len(v))
    trace = {"m.x": pad(5, 6, 7, 0, 9), "m.s": pad(1, 1, 1, 0, 0),
             "m.y": pad(0, 7, 6, 9 if bad else 5), "m.r": pad(0, 1, 1, 1)}
    pb = _prove(compiled, _witness(b, compiled, trace), 8)
    if bad:
        with pytest.raises(oracle.VerifyError, match="do not multiply to one"):
            oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)
    else:
        oracle.verify(compiled.words, pb, 8, product_buses=compiled.product_buses)


@pytest.mark.parametrize("bad", [False, True])
def test_lookup_source_and_target_in_one_module(bad):
    """lookup_test.go TestSourceAndTargetShareColumn: source and table in one
    module give one logup column and one total; a source value outside the
    table is refused by the prover."""
    from loom_b200.program import col, lookup
    n = 8
    b = _one_module(n)
    totals = lookup(b, [(col("m.s"), "m")], [(col("m.t"), "m")])
    compiled = b.compile()
    assert compiled.logup_buses == [list(totals)] and len(totals) == 1
    src = [(3 * i) % n for i in range(n)]
    if bad:
        src[2] = 100
    wit = _witness(b, compiled, {"m.t": list(range(n)), "m.s": src})
    if bad:
        with pytest.raises(RuntimeError, match="not in the table"):
            _prove(compiled, wit, 8)
    else:
        oracle.verify(compiled.words, _prove(compiled, wit, 8), 8, compiled.logup_buses)


def _exposed_offsets(pb):
    """Byte offset of the first word of each exposed value's first entry
    (the encoding: backend string, then per name: string, entry count,
    entries of index, field kind and six words)."""
    o = 4 + struct.unpack_from(">I", pb, 0)[0]
    count = struct.unpack_from(">I", pb, o)[0]
    o += 4
    offs = {}
    for _ in range(count):
        ln = struct.unpack_from(">I", pb, o)[0]
        name = pb[o + 4:o + 4 + ln].decode()
        o += 4 + ln
        entries = struct.unpack_from(">I", pb, o)[0]
        o += 4
        offs[name] = o + 8
        o += entries * 32
    return offs


@pytest.mark.parametrize("bad", [False, True])
def test_batched_cyclic_lookup(bad):
    """lookup_test.go TestBatchedCyclicLookup and
    TestBatchedCyclicLookupRejectsMissingValue: four sources of module m
    looked up in one table share one logup column of m; the two exposed
    totals are bound to the transcript, so changing either is rejected; a
    source value outside the table is refused by the prover."""
    from loom_b200.program import Builder, Module, col, lookup
    n = 16
    b = Builder()
    b.add_module(Module("m", n))
    b.add_module(Module("tab", n))
    totals = lookup(b, [(col(f"m.s{k}"), "m") for k in range(4)], [(col("tab.t"), "tab")])
    assert [t.split(".")[0] for t in totals] == ["m", "tab"]  # one logup column per module
    compiled = b.compile()
    s2 = [3] * n
    if bad:
        s2[5] = 100
    trace = {"tab.t": list(range(n)), "m.s0": list(range(n)), "m.s1": [n - 1 - i for i in range(n)],
             "m.s2": s2, "m.s3": [i // 2 for i in range(n)]}
    wit = _witness(b, compiled, trace)
    if bad:
        with pytest.raises(RuntimeError, match="not in the table"):
            _prove(compiled, wit, 8)
        return
    pb = _prove(compiled, wit, 8)
    oracle.verify(compiled.words, pb, 8, compiled.logup_buses)
    offs = _exposed_offsets(pb)
    assert len(offs) == 2 and set(proof.decode(pb).exposed) == set(offs)
    for name, at in offs.items():
        tampered = bytearray(pb)
        struct.pack_into(">I", tampered, at, (struct.unpack_from(">I", pb, at)[0] + 1) % F.P)
        with pytest.raises(oracle.VerifyError):
            oracle.verify(compiled.words, bytes(tampered), 8, compiled.logup_buses)


@pytest.mark.parametrize("bad", [False, True])
def test_lookup_selectors(bad):
    """lookups_test.go TestLookupsSelectors: two selected sources of module a
    into one selected table (one logup column per module); unselected source rows
    hold anything; a selected source equal to an unselected table row is
    refused."""
    from loom_b200.program import Builder, Module, col, lookup_tuple
    n = 8
    b = Builder()
    for name in ("a", "tab"):
        b.add_module(Module(name, n))
    totals = lookup_tuple(b, [([col("a.s0")], "a"), ([col("a.s1")], "a")], [([col("tab.t")], "tab")],
                          sel_s=[col("a.sels0"), col("a.sels1")], sel_t=[col("tab.sel")])
    compiled = b.compile()
    assert compiled.logup_buses == [list(totals)] and [t.split(".")[0] for t in totals] == ["a", "tab"]
    pad = lambda *v: list(v) + [0] * (n - len(v))
    trace = {"tab.t": pad(10, 11, 12, 13), "tab.sel": pad(1, 1, 1, 0),
             "a.s0": pad(10, 99, 12, 12), "a.sels0": pad(1, 0, 1, 1),
             "a.s1": pad(11, 77, 13 if bad else 11), "a.sels1": pad(1, 0, 1)}
    wit = _witness(b, compiled, trace)
    if bad:
        with pytest.raises(RuntimeError, match="not in the table"):
            _prove(compiled, wit, 8)
    else:
        oracle.verify(compiled.words, _prove(compiled, wit, 8), 8, compiled.logup_buses)


@pytest.mark.parametrize("bad", [False, True])
def test_lookups_share_target(bad):
    """lookups_test.go TestLookupsShareTarget (grouped form): a.s0, a.s1 and
    b.s looked up in one table give one bus with three totals (a, b, tab),
    the two sources of module a batched in one logup column; a source value
    outside the table is refused."""
    from loom_b200.program import Builder, Module, col, lookup
    n = 8
    b = Builder()
    for name in ("a", "b", "tab"):
        b.add_module(Module(name, n))
    totals = lookup(b, [(col("a.s0"), "a"), (col("a.s1"), "a"), (col("b.s"), "b")], [(col("tab.t"), "tab")])
    compiled = b.compile()
    assert compiled.logup_buses == [list(totals)] and [t.split(".")[0] for t in totals] == ["a", "b", "tab"]
    bs = [5] * n
    if bad:
        bs[3] = 100
    wit = _witness(b, compiled, {"tab.t": list(range(n)), "a.s0": [i // 2 for i in range(n)],
                                 "a.s1": [n - 1 - i for i in range(n)], "b.s": bs})
    if bad:
        with pytest.raises(RuntimeError, match="not in the table"):
            _prove(compiled, wit, 8)
    else:
        oracle.verify(compiled.words, _prove(compiled, wit, 8), 8, compiled.logup_buses)

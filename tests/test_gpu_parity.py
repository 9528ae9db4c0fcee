"""GPU parity: every CUDA entry point against the CPU oracle, through the C ABI.

Integer/field work, so the bar is bit-exact equality.  Sizes are ones the
oracle finishes in seconds; workloads too large for the oracle (the mixed
40-module lookup program, 2^20-row modules) are covered by size-independent
properties: batched == plain bytes, a constant FRI final polynomial, balanced
logup totals.
"""
import numpy as np
import pytest

import oracle
from loom_b200 import LoomError, field as F, plonk, proof

pytestmark = pytest.mark.gpu


def rnd(shape, seed):
    return np.random.Generator(np.random.PCG64(seed)).integers(0, F.P, shape, dtype=np.uint64).astype(np.uint32)


def test_poseidon2_permutation(ctx):
    canon = rnd((257, 24), 1)
    canon[0] = 0
    got = F.from_mont(ctx.poseidon2_permute(F.to_mont(canon)))
    for i in range(canon.shape[0]):
        assert np.array_equal(got[i], oracle.p2_permute(canon[i], 24)), i


@pytest.mark.parametrize("logn", [1, 2, 5, 8, 10, 12, 13, 14])
def test_rs_encode(ctx, logn):
    cols = F.to_mont(rnd((3, 1 << logn), logn))
    got = ctx.rs_encode(cols)
    for i in range(3):
        assert np.array_equal(got[i], oracle.rs_encode(cols[i], 4 << logn)), (logn, i)


def test_rs_encode_edge_values(ctx):
    n = 1 << 9
    cols = np.stack([np.zeros(n), np.full(n, F.P - 1), np.arange(n) % 2]).astype(np.uint32)
    cols = F.to_mont(cols)
    got = ctx.rs_encode(cols)
    for i in range(cols.shape[0]):
        assert np.array_equal(got[i], oracle.rs_encode(cols[i], 4 * n))


@pytest.mark.parametrize("shape", [
    [(1 << 10, 3, 0)],
    [(1 << 8, 0, 1)],
    [(1 << 10, 2, 1), (1 << 10, 1, 0), (1 << 8, 4, 2), (1 << 10, 0, 1), (1 << 6, 1, 0), (1 << 9, 2, 0)],
    [(2, 1, 0), (2, 0, 1)],
])
def test_commit_root(ctx, shape):
    groups = []
    for gi, (n, nb, ne) in enumerate(shape):
        groups.append({"rows": n,
                       "base": [F.to_mont(rnd(n, 100 * gi + k)) for k in range(nb)],
                       "ext": [F.to_mont(rnd((n, 6), 100 * gi + 50 + k)) for k in range(ne)]})
    assert np.array_equal(ctx.commit_root(groups), oracle.commit(groups))


def test_merkle_injections(ctx):
    leaves = F.to_mont(rnd((64, 8), 7))
    inj = [F.to_mont(rnd((64, 8), 8)), F.to_mont(rnd((64, 8), 9)), F.to_mont(rnd((16, 8), 10)),
           F.to_mont(rnd((2, 8), 11)), F.to_mont(rnd((1, 8), 12)), F.to_mont(rnd((1, 8), 13))]
    assert np.array_equal(ctx.merkle_root(leaves, inj), oracle.merkle_root(leaves, inj))
    assert np.array_equal(ctx.merkle_root(leaves[:1]), oracle.merkle_root(leaves[:1]))


def test_merkle_injection_order_and_schedule_checks(ctx):
    """Same-width injections do not commute (the GPU agrees with the oracle
    either way), and a schedule merkle.NewWithInjections rejects (a width
    that grows, exceeds the leaves or is not a power of two) is refused."""
    leaves = F.to_mont(rnd((8, 8), 10))
    a, b = F.to_mont(rnd((4, 8), 11)), F.to_mont(rnd((4, 8), 12))
    ab, ba = ctx.merkle_root(leaves, [a, b]), ctx.merkle_root(leaves, [b, a])
    assert not np.array_equal(ab, ba)
    assert np.array_equal(ab, oracle.merkle_root(leaves, [a, b]))
    assert np.array_equal(ba, oracle.merkle_root(leaves, [b, a]))
    for widths in ([4, 8], [16], [3], [0]):
        with pytest.raises(LoomError, match="injection"):
            ctx.merkle_root(leaves, [F.to_mont(rnd((w, 8), 20 + w)) for w in widths])


@pytest.mark.parametrize("logn", [1, 4, 11, 16])
def test_fri_fold(ctx, logn):
    layer = F.to_mont(rnd((1 << logn, 6), logn))
    alpha = F.to_mont(rnd(6, 99))
    assert np.array_equal(ctx.fri_fold(layer, alpha), oracle.fri_fold(layer, alpha))


def _prove_both(ctx, n_inst, n, q, seed):
    compiled, wit = plonk.build(n_inst, n, seed=seed)
    mont = [F.to_mont(w) for w in wit]
    return ctx.prove(compiled.words, mont, q), oracle.prove(compiled.words, mont, q)


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("n_inst,logn,q", [(1, 4, 1), (2, 10, 16), (4, 12, 200), (3, 13, 7), (5, 9, 3)])
def test_prove_bytes_equal_oracle(ctx, n_inst, logn, q, batched):
    ctx.set_batched(batched)
    try:
        got, want = _prove_both(ctx, n_inst, 1 << logn, q, seed=0x10AD + logn)
    finally:
        ctx.set_batched(True)
    assert len(got) == len(want)
    assert got == want
    p = proof.decode(got)
    assert all(v == p.final_poly[0] for v in p.final_poly)


@pytest.mark.parametrize("batched", [True, False])
def test_prove_uneven_modules(ctx, batched):
    from loom_b200.program import Builder, Module, col, copy_constraint
    # modules of 2^8, 2^10 and 2^11 rows in one program
    b = Builder()
    trace = {}
    for i, logn in enumerate([10, 8, 11, 8]):
        n = 1 << logn
        m = Module(f"plonk_{i}", n)
        L, R, O = col(f"L_{i}"), col(f"R_{i}"), col(f"O_{i}")
        QL, QR, QM, QO, QK = (col(f"{s}_{i}") for s in ("QL", "QR", "QM", "QO", "QK"))
        m.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
        b.add_module(m)
        w, S = plonk.instance_witness(n, 5, i)
        trace.update(w)
        copy_constraint(b, m.name, [L, R, O], S, f"plonk.S_{i}")
    trace.update(b.generated)
    compiled = b.compile()
    mont = [F.to_mont(trace[name]) for (name, _, _) in compiled.witness_columns]
    ctx.set_batched(batched)
    try:
        got = ctx.prove(compiled.words, mont, 20)
    finally:
        ctx.set_batched(True)
    assert got == oracle.prove(compiled.words, mont, 20)


@pytest.mark.parametrize("mapping", [1, 6])
def test_leaf_mappings_agree(ctx, mapping):
    compiled, wit = plonk.build(3, 1 << 11, seed=21)
    mont = [F.to_mont(w) for w in wit]
    ctx.set_leaf_mapping(mapping)
    try:
        got = ctx.prove(compiled.words, mont, 9)
    finally:
        ctx.set_leaf_mapping(0)
    assert got == oracle.prove(compiled.words, mont, 9)


def test_repeated_proves_identical(ctx):
    compiled, wit = plonk.build(2, 1 << 9, seed=3)
    mont = [F.to_mont(w) for w in wit]
    a = ctx.prove(compiled.words, mont, 8)
    b = ctx.prove(compiled.words, mont, 8)
    assert a == b


def test_prove_into_caller_buffer(ctx):
    """The proof lands in the caller's buffer (exact size, and larger); a
    buffer one byte short is refused with LG_ERR_BUFFER and the needed size,
    and the context keeps that proof for lg_last_proof (prove() re-reads it)."""
    compiled, wit = plonk.build(2, 1 << 9, seed=5)
    mont = [F.to_mont(w) for w in wit]
    ref = ctx.prove(compiled.words, mont, 8)
    exact = bytearray(len(ref))
    assert ctx.prove_into(exact, compiled.words, mont, 8) == len(ref)
    assert bytes(exact) == ref
    big = np.zeros(len(ref) + 4096, dtype=np.uint8)
    n = ctx.prove_into(big, compiled.words, mont, 8)
    assert n == len(ref) and big[:n].tobytes() == ref and not big[n:].any()
    with pytest.raises(LoomError) as e:
        ctx.prove_into(bytearray(len(ref) - 1), compiled.words, mont, 8)
    assert e.value.code == 5 and str(len(ref)) in str(e.value)
    ctx._proof_cap = 16  # force prove() through LG_ERR_BUFFER + lg_last_proof
    assert ctx.prove(compiled.words, mont, 8) == ref


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("sizes,q", [([6, 5, 7, 4], 8), ([10, 12, 9, 11, 10], 24)])
def test_prove_lookup_equals_oracle(ctx, sizes, q, batched):
    """Uneven modules with a range lookup (logup into a shared 2^8 table):
    multiplicities, cyclic logup columns, exposed totals and their binding."""
    compiled, wit = plonk.build_mixed(sizes, seed=sum(sizes))
    mont = [F.to_mont(w) for w in wit]
    ctx.set_batched(batched)
    try:
        got = ctx.prove(compiled.words, mont, q)
    finally:
        ctx.set_batched(True)
    assert got == oracle.prove(compiled.words, mont, q)
    assert proof.decode(got).exposed


def test_mixed_lookup_full_size_properties(ctx):
    """The batched form at full size: 40 modules with log2 rows 10-20
    (seeded), plonk gates + copy constraint + range lookup.  Too large for
    the oracle, so checked through size-independent properties: batched and
    plain proofs are the same bytes, the FRI final polynomial is constant
    (every constraint holds) and the logup totals balance."""
    sizes = plonk.mixed_sizes(40, 10, 20, 0xC4)
    compiled, wit = plonk.build_mixed(sizes, seed=0xC4)
    mont = [F.to_mont(w) for w in wit]
    a = ctx.prove(compiled.words, mont, 32)
    ctx.set_batched(False)
    try:
        b = ctx.prove(compiled.words, mont, 32)
    finally:
        ctx.set_batched(True)
    assert a == b
    p = proof.decode(a)
    assert all(v == p.final_poly[0] for v in p.final_poly)
    bus = [0] * 6
    for ents in p.exposed.values():
        for (_, _, e) in ents:
            bus = [(x + y) % F.P for x, y in zip(bus, e)]
    assert bus == [0] * 6 and len(p.exposed) == 80
    oracle.verify(compiled.words, a, 32, compiled.logup_buses)


def test_mixed_lookup_full_size_equals_oracle_digest(ctx):
    """The batched form at full size against the oracle, byte for byte: 40
    modules with log2 rows 10-20 drawn with seed 0xC4, plonk gates, a copy
    constraint and a range lookup, 200 queries.  The oracle's proof (several
    minutes on the CPU) is recorded as its length and SHA-256 by
    tests/golden/make_c4_digest.py; batched and plain GPU proofs must hash
    to the same."""
    import hashlib
    import json
    import os
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c4_mixed_lookup_digest.json")))
    sizes = plonk.mixed_sizes(40, 10, 20, fx["seed"])
    assert sizes == fx["log_sizes"]
    compiled, wit = plonk.build_mixed(sizes, seed=fx["seed"])
    assert hashlib.sha256(compiled.words.astype("<u4").tobytes()).hexdigest() == fx["program_sha256"]
    mont = [F.to_mont(w) for w in wit]
    for batched in (True, False):
        ctx.set_batched(batched)
        try:
            got = ctx.prove(compiled.words, mont, fx["queries"])
        finally:
            ctx.set_batched(True)
        assert len(got) == fx["proof_len"], batched
        assert hashlib.sha256(got).hexdigest() == fx["proof_sha256"], batched


@pytest.mark.parametrize("permuted", [True, False])
@pytest.mark.parametrize("logn", [6, 12])
def test_prove_running_ratio_equals_oracle(ctx, logn, permuted):
    compiled, wit, end = plonk.build_with_ratio(1 << logn, seed=logn, permuted=permuted)
    mont = [F.to_mont(w) for w in wit]
    got = ctx.prove(compiled.words, mont, 12)
    assert got == oracle.prove(compiled.words, mont, 12)
    (idx, kind, e), = proof.decode(got).exposed[end]
    assert (tuple(e) == (1, 0, 0, 0, 0, 0)) == permuted
    if permuted:
        oracle.verify(compiled.words, got, 12, product_buses=compiled.product_buses)
    else:
        with pytest.raises(oracle.VerifyError, match="do not multiply to one"):
            oracle.verify(compiled.words, got, 12, product_buses=compiled.product_buses)


@pytest.mark.parametrize("balanced", [True, False])
@pytest.mark.parametrize("logn", [6, 11])
def test_prove_bus_equals_oracle(ctx, logn, balanced):
    """arguments.Bus (width-2 tuples, selectors, two modules): running-ratio
    columns packed by degree, product bus over their ends."""
    compiled, wit, ends = plonk.build_with_bus(1 << logn, seed=logn, balanced=balanced)
    mont = [F.to_mont(w) for w in wit]
    got = ctx.prove(compiled.words, mont, 12)
    assert got == oracle.prove(compiled.words, mont, 12)
    if balanced:
        oracle.verify(compiled.words, got, 12, product_buses=compiled.product_buses)
    else:
        with pytest.raises(oracle.VerifyError, match="do not multiply to one"):
            oracle.verify(compiled.words, got, 12, product_buses=compiled.product_buses)


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("n_inst,logn", [(2, 6), (3, 11)])
def test_prove_with_setup_equals_oracle(ctx, n_inst, logn, batched):
    """setup.Setup then Prove: the selectors, copy permutation and identity
    columns precommitted once (lg_setup); the root equals the oracle's, the
    proofs equal the oracle's byte for byte on every prove that reuses the
    precommit, and the verifier accepts them under that key."""
    compiled, wit, setup = plonk.build_with_setup(n_inst, 1 << logn, seed=logn)
    wm = [F.to_mont(w) for w in wit]
    sm = [F.to_mont(x) for x in setup]
    root = ctx.setup(compiled.words, sm)
    want_root = oracle.setup_root(compiled.words, sm)
    assert F.from_mont(root).tolist() == want_root.tolist()
    ctx.set_batched(batched)
    try:
        got = ctx.prove(compiled.words, wm, 12)
        again = ctx.prove(compiled.words, wm, 12)
    finally:
        ctx.set_batched(True)
    assert got == again == oracle.prove(compiled.words, wm, 12, sm)
    oracle.verify(compiled.words, got, 12, setup_root=want_root)


@pytest.mark.parametrize("batched", [True, False])
@pytest.mark.parametrize("logn", [6, 12])
def test_prove_tuple_lookup_equals_oracle(ctx, logn, batched):
    """arguments.CLookupUnionTuple on the GPU: width-2 tuples from two modules
    with selectors of weight 1 and 2 into a table with selectors 0, 1, 3 and
    repeated tuples (device hash table on tuples, 64-bit weights)."""
    compiled, wit = plonk.build_with_tuple_lookup(1 << logn, seed=logn)
    mont = [F.to_mont(w) for w in wit]
    ctx.set_batched(batched)
    try:
        got = ctx.prove(compiled.words, mont, 12)
    finally:
        ctx.set_batched(True)
    assert got == oracle.prove(compiled.words, mont, 12)
    oracle.verify(compiled.words, got, 12, compiled.logup_buses)


def test_prove_tuple_lookup_missing_tuple_is_refused(ctx):
    compiled, wit = plonk.build_with_tuple_lookup(1 << 6, present=False)
    with pytest.raises(LoomError) as e:
        ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 4)
    assert e.value.code == 1 and "not in its table" in str(e.value)


def test_prove_without_setup_is_refused(ctx):
    compiled, wit, setup = plonk.build_with_setup(1, 1 << 5, seed=3)
    with pytest.raises(LoomError) as e:
        ctx.prove(compiled.words, [F.to_mont(w) for w in wit], 4)
    assert e.value.code == 1 and "lg_setup" in str(e.value)


def test_prove_lookup_value_outside_table_is_refused(ctx):
    compiled, wit = plonk.build_mixed([6, 5], seed=4)
    mont = [F.to_mont(w) for w in wit]
    i = [c[0] for c in compiled.witness_columns].index("RC_1")
    mont[i] = mont[i].copy()
    mont[i][7] = F.to_mont(np.array([1000], dtype=np.uint32))[0]
    with pytest.raises(LoomError) as e:
        ctx.prove(compiled.words, mont, 4)
    assert e.value.code == 1 and "not in its table" in str(e.value)


def test_tuning_never_changes_proofs(ctx):
    """Launch-shape values at the ends of their ranges give the same proof
    bytes; invalid names and values are refused."""
    compiled, wit = plonk.build(3, 1 << 10, seed=9)
    mont = [F.to_mont(w) for w in wit]
    defaults = ctx.tuning()
    ref = ctx.prove(compiled.words, mont, 16)
    try:
        for params in ({"merkle_tail": 2, "merkle_subtree": 2, "p2_leaf_min_per_sm": 0, "p2_node_min_per_sm": 0,
                        "p2_inject_min_per_sm": 0, "inject_block": 1024, "leaf_block": 32, "lde_split": 0,
                        "lde_fwd_threads": 256, "fri_tail_leaves": 0, "quotient_jit": 0, "upload_split": 0},
                       {"merkle_tail": 1024, "merkle_subtree": 1024, "p2_leaf_min_per_sm": 1 << 20,
                        "p2_node_min_per_sm": 1 << 20, "p2_inject_min_per_sm": 1 << 20, "inject_block": 32,
                        "leaf_block": 1024, "lde_split": 1, "lde_fwd_threads": 1024, "fri_tail_leaves": 65536},
                       {"merkle_tail": 64, "merkle_subtree": 0, "p2_leaf_min_per_sm": 128,
                        "p2_node_min_per_sm": 512, "inject_block": 32, "leaf_block": 128},
                       {"merkle_tail": 4, "merkle_subtree": 8, "p2_leaf_min_per_sm": 128,
                        "p2_node_min_per_sm": 512, "inject_block": 32, "leaf_block": 128}):
            ctx.apply_tuning(params)
            got = ctx.tuning()
            assert {k: got[k] for k in params} == params
            assert ctx.prove(compiled.words, mont, 16) == ref
    finally:
        ctx.apply_tuning(defaults)
    for name, value in (("merkle_tail", 48), ("merkle_tail", 2048), ("merkle_subtree", 1), ("merkle_subtree", 48),
                        ("leaf_block", 16), ("lde_split", 2), ("lde_fwd_threads", 128), ("fri_tail_leaves", 3), ("quotient_jit", 2), ("upload_split", 2),
                        ("no_such", 1)):
        with pytest.raises(LoomError) as e:
            ctx.set_tuning(name, value)
        assert e.value.code == 1
    assert ctx.tuning() == defaults


def test_unsupported_hash_backend(ctx):
    compiled, wit = plonk.build(1, 1 << 4, seed=1)
    mont = [F.to_mont(w) for w in wit]
    for hb in ("sha256", "blake3"):
        with pytest.raises(LoomError) as e:
            ctx.prove(compiled.words, mont, 4, hash_backend=hb)
        assert e.value.code == 4


def test_malformed_program(ctx):
    compiled, wit = plonk.build(1, 1 << 4, seed=1)
    mont = [F.to_mont(w) for w in wit]
    bad = compiled.words.copy()
    bad[0] ^= 1
    with pytest.raises(LoomError) as e:
        ctx.prove(bad, mont, 4)
    assert e.value.code == 1
    with pytest.raises(LoomError):
        ctx.prove(compiled.words[:10], mont, 4)
    # the context stays usable after errors
    assert ctx.prove(compiled.words, mont, 4) == oracle.prove(compiled.words, mont, 4)


@pytest.mark.parametrize("n", [1, 2, 7, 2048, 2049, 5000, 1 << 14])
def test_grand_product(ctx, n):
    num = F.to_mont(rnd((n, 6), n))
    den = F.to_mont(rnd((n, 6), n + 1))
    assert np.array_equal(ctx.grand_product(num, den), oracle.grand_product(num, den))


@pytest.mark.parametrize("logn,cols", [(15, 3), (16, 2), (17, 1), (18, 1), (20, 1), (21, 1), (22, 1)])
def test_rs_encode_large(ctx, logn, cols):
    c = F.to_mont(rnd((cols, 1 << logn), 300 + logn))
    got = ctx.rs_encode(c)
    for i in range(cols):
        assert np.array_equal(got[i], oracle.rs_encode(c[i], 4 << logn)), (logn, i)


@pytest.mark.parametrize("tail", [0, 2, 512, 65536])
def test_fri_tail_block_gives_identical_proofs(ctx, tail):
    """The last FRI rounds in one block (k_fri_tail) or one launch per step:
    the same proof, including levels that enter inside the tail (modules of
    uneven sizes)."""
    compiled, wit = plonk.build_mixed([12, 5, 9, 7, 4], seed=23)
    mont = [F.to_mont(w) for w in wit]
    saved = ctx.get_tuning("fri_tail_leaves")
    try:
        ctx.set_tuning("fri_tail_leaves", tail)
        got = ctx.prove(compiled.words, mont, 20)
    finally:
        ctx.set_tuning("fri_tail_leaves", saved)
    assert got == oracle.prove(compiled.words, mont, 20)


@pytest.mark.parametrize("build", ["plonk", "mixed_lookup"])
def test_compiled_constraint_kernels_give_identical_proofs(ctx, build):
    """The quotient's constraint bytecode compiled to kernels at run time
    (tuning quotient_jit = 1, the default) against the bytecode interpreter
    (0): the same proof, equal to the oracle's, with compiled kernels in use."""
    from loom_b200 import _lib
    L = _lib.load()
    if build == "plonk":
        compiled, wit = plonk.build(3, 1 << 9, seed=31)
    else:
        compiled, wit = plonk.build_mixed([7, 5, 9, 5], seed=11)
    mont = [F.to_mont(w) for w in wit]
    saved = ctx.get_tuning("quotient_jit")
    try:
        ctx.set_tuning("quotient_jit", 0)
        interp = ctx.prove(compiled.words, mont, 16)
        ctx.set_tuning("quotient_jit", 1)
        jit = ctx.prove(compiled.words, mont, 16)
    finally:
        ctx.set_tuning("quotient_jit", saved)
    assert jit == interp == oracle.prove(compiled.words, mont, 16)
    assert L.lg_jit_kernels() >= 1


@pytest.mark.parametrize("build", ["plonk", "mixed_lookup"])
def test_split_witness_upload_gives_identical_proofs(ctx, build):
    """A host witness's columns that round 0 does not commit go up on a second
    stream while round 0 runs (tuning upload_split = 1, the default; a first
    round with witness steps waits for all of them): the proof of a
    device-resident witness with the split and without, from pageable arrays
    and from one page-locked buffer whose columns are adjacent."""
    import torch
    if build == "plonk":
        compiled, wit = plonk.build(5, 1 << 9, seed=41)
    else:
        compiled, wit = plonk.build_mixed([7, 5, 9, 5, 8], seed=13)
    mont = [np.ascontiguousarray(F.to_mont(w), dtype=np.uint32) for w in wit]
    dev = [torch.from_numpy(m.astype(np.int64)).to(torch.int32).cuda() for m in mont]
    ref = ctx.prove(compiled.words, [t.data_ptr() for t in dev], 16, on_device=True)
    pinned = torch.empty(sum(m.size for m in mont), dtype=torch.int32).pin_memory()
    flat = pinned.numpy().view(np.uint32)
    views, off = [], 0
    for m in mont:
        flat[off:off + m.size] = m
        views.append(flat[off:off + m.size])
        off += m.size
    saved = ctx.get_tuning("upload_split")
    try:
        for split in (1, 0):
            ctx.set_tuning("upload_split", split)
            assert ctx.prove(compiled.words, mont, 16) == ref
            assert ctx.prove(compiled.words, views, 16) == ref
    finally:
        ctx.set_tuning("upload_split", saved)
    assert ref == oracle.prove(compiled.words, mont, 16)


def test_lde_launch_shapes_give_identical_results(ctx):
    """The LDE's launch structure is a tuning choice: fused (one block per
    lane) or split (inverse launch, then one block per lane and coset, with
    256, 512 or 1024 threads); outputs and proofs must not depend on it."""
    cols = F.to_mont(rnd((5, 1 << 14), 77))
    want = [oracle.rs_encode(cols[i], 4 << 14) for i in range(5)]
    compiled, wit = plonk.build(3, 1 << 12, seed=9)
    mont = [F.to_mont(w) for w in wit]
    base = ctx.prove(compiled.words, mont, 16)
    saved = {k: ctx.get_tuning(k) for k in ("lde_split", "lde_fwd_threads")}
    try:
        for split, thr in ((0, 512), (1, 256), (1, 512), (1, 1024)):
            ctx.set_tuning("lde_split", split)
            ctx.set_tuning("lde_fwd_threads", thr)
            got = ctx.rs_encode(cols)
            assert all(np.array_equal(got[i], want[i]) for i in range(5)), (split, thr)
            assert ctx.prove(compiled.words, mont, 16) == base, (split, thr)
    finally:
        ctx.apply_tuning(saved)
    assert base == oracle.prove(compiled.words, mont, 16)


def test_commit_root_large_and_small(ctx):
    groups = [{"rows": 1 << 10, "base": [F.to_mont(rnd(1 << 10, 5))]},
              {"rows": 1 << 16, "base": [F.to_mont(rnd(1 << 16, 6)), F.to_mont(rnd(1 << 16, 7))],
               "ext": [F.to_mont(rnd((1 << 16, 6), 8))]},
              {"rows": 1 << 15, "ext": [F.to_mont(rnd((1 << 15, 6), 9))]}]
    assert np.array_equal(ctx.commit_root(groups), oracle.commit(groups))


def test_prove_large_module(ctx):
    from loom_b200.program import Builder, Module, col, copy_constraint
    b = Builder()
    trace = {}
    for i, logn in enumerate([15, 10]):
        n = 1 << logn
        m = Module(f"plonk_{i}", n)
        L, R, O = col(f"L_{i}"), col(f"R_{i}"), col(f"O_{i}")
        QL, QR, QM, QO, QK = (col(f"{s}_{i}") for s in ("QL", "QR", "QM", "QO", "QK"))
        m.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
        b.add_module(m)
        w, S = plonk.instance_witness(n, 17, i)
        trace.update(w)
        copy_constraint(b, m.name, [L, R, O], S, f"plonk.S_{i}")
    trace.update(b.generated)
    compiled = b.compile()
    mont = [F.to_mont(trace[name]) for (name, _, _) in compiled.witness_columns]
    got = ctx.prove(compiled.words, mont, 4)
    assert got == oracle.prove(compiled.words, mont, 4)
    oracle.verify(compiled.words, got, 4)


def test_verifier_accepts_gpu_proofs_and_rejects_false_ones(ctx):
    """GPU proofs too large for the oracle prover at these query counts go
    through the oracle's verifier; a GPU proof of a violated gate does not
    verify."""
    compiled, wit = plonk.build(8, 1 << 13, seed=0x5EED)
    mont = [F.to_mont(w) for w in wit]
    got = ctx.prove(compiled.words, mont, 200)
    oracle.verify(compiled.words, got, 200)
    names = [n for (n, _, _) in compiled.witness_columns]
    bad = [m.copy() for m in mont]
    i = names.index("O_5")
    bad[i][100] = F.to_mont(np.array([(int(F.from_mont(bad[i][100:101])[0]) + 1) % F.P], dtype=np.uint32))[0]
    with pytest.raises(oracle.VerifyError, match="AIR relation"):
        oracle.verify(compiled.words, ctx.prove(compiled.words, bad, 200), 200)


@pytest.mark.parametrize("cols,logr", [(1, 3), (5, 10), (37, 12)])
def test_deep_quotient(ctx, cols, logr):
    lde = F.to_mont(rnd((cols, 1 << logr), cols))
    alpha, z = F.to_mont(rnd(6, 1)), F.to_mont(rnd(6, 2))
    values = F.to_mont(rnd((cols, 6), 3))
    assert np.array_equal(ctx.deep_quotient(lde, alpha, z, values), oracle.deep_quotient(lde, alpha, z, values))

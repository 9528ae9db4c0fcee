"""The oracle against the relations the reference's own tests check
(internal/reedsolomon/rs_eval_test.go, internal/merkle/injection_test.go,
internal/hash/hash_test.go, internal/fri/fold_bitrev_test.go) and
prove-level invariants (low-degree final polynomial, vanishing quotient
chunk, tamper sensitivity)."""
import numpy as np
import pytest

import oracle
from loom_b200 import field as F, plonk, proof

P = F.P


def rnd(shape, seed):
    return np.random.Generator(np.random.PCG64(seed)).integers(0, P, shape, dtype=np.uint64).astype(np.uint32)


def bitrev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("logn", [1, 3, 6])
def test_rs_encode_equals_direct_evaluation(logn):
    # rs_eval_test.go: encode == P evaluated at the bit-reversed roots
    n = 1 << logn
    vals = rnd(n, logn).tolist()
    w = F.root_of_unity(n)
    ninv = pow(n, P - 2, P)
    winv = pow(w, P - 2, P)
    coeffs = [sum(vals[j] * pow(winv, j * k, P) for j in range(n)) * ninv % P for k in range(n)]
    big = 4 * n
    W = F.root_of_unity(big)
    got = F.from_mont(oracle.rs_encode(F.to_mont(vals), big)).tolist()
    for r in range(big):
        x = pow(W, bitrev(r, logn + 2), P)
        assert got[r] == sum(c * pow(x, k, P) for k, c in enumerate(coeffs)) % P


def _node(l, r):
    st = [0x4E4F4445] + [0] * 7 + list(l) + list(r)
    return oracle.p2_permute(st, 24)[:8].tolist()


def test_merkle_injections_match_naive_root():
    # injection_test.go: schedule vs a naive reference root
    leaves = [rnd(8, i).tolist() for i in range(8)]
    inj = [[rnd(8, 100 + i).tolist() for i in range(8)], [rnd(8, 200 + i).tolist() for i in range(2)],
           [rnd(8, 300).tolist()]]
    level = [_node(leaves[i], inj[0][i]) for i in range(8)]
    widths = [len(x) for x in inj]
    nxt = 1
    while len(level) > 1:
        level = [_node(level[2 * i], level[2 * i + 1]) for i in range(len(level) // 2)]
        while nxt < len(inj) and widths[nxt] == len(level):
            level = [_node(level[j], inj[nxt][j]) for j in range(len(level))]
            nxt += 1
    got = oracle.merkle_root(F.to_mont(np.array(leaves)), [F.to_mont(np.array(x)) for x in inj])
    assert F.from_mont(got).tolist() == level[0]


def test_same_width_injection_order_matters():
    # injection_test.go TestSameWidthOrderMatters: the order of two injections
    # of one width is part of the commitment
    leaves = F.to_mont(rnd((8, 8), 10))
    a, b = F.to_mont(rnd((4, 8), 11)), F.to_mont(rnd((4, 8), 12))
    assert not np.array_equal(oracle.merkle_root(leaves, [a, b]), oracle.merkle_root(leaves, [b, a]))


@pytest.mark.parametrize("widths", [[4, 8], [16], [3], [0]])
def test_bad_injection_schedule_is_rejected(widths):
    # injection_test.go TestInjectionScheduleValidation / validateInjections
    # (internal/merkle/tree.go:140-160): widths must be powers of two, at most
    # the leaves, and must not increase
    leaves = F.to_mont(rnd((8, 8), 10))
    inj = [F.to_mont(rnd((w, 8), 20 + w)) for w in widths]
    with pytest.raises(ValueError, match="injection"):
        oracle.merkle_root(leaves, inj)


def _py_sponge(elems):
    state = [0] * 24
    block = []
    wrote = False
    for x in elems:
        block.append(x)
        if len(block) == 16:
            state[:16] = block
            state = oracle.p2_permute(state, 24).tolist()
            block, wrote = [], True
    if not wrote and not block:
        return [0] * 8
    if block:
        state[:len(block)] = block
        state = oracle.p2_permute(state, 24).tolist()
    return state[:8]


@pytest.mark.parametrize("n", [0, 1, 15, 16, 17, 32, 51])
def test_sponge_matches_reference_sponge(n):
    # hash_test.go: sponge vs an in-test reference sponge (overwrite, no padding)
    elems = rnd(n, n).tolist()
    assert F.from_mont(oracle.sponge(F.to_mont(np.array(elems, dtype=np.uint32)))).tolist() == _py_sponge(elems)


def _e6_mul_py(x, y):
    # recursion/e6.go:24-53 schoolbook over E2 with u^2 = 3, v^3 = u + 1
    def m2(a0, a1, b0, b1):
        return (a0 * b0 + 3 * a1 * b1) % P, (a0 * b1 + a1 * b0) % P

    def xi(p0, q0):
        return (p0 + 3 * q0) % P, (p0 + q0) % P
    pr = {(i, j): m2(x[2 * i], x[2 * i + 1], y[2 * j], y[2 * j + 1]) for i in range(3) for j in range(3)}
    t0 = xi((pr[1, 2][0] + pr[2, 1][0]) % P, (pr[1, 2][1] + pr[2, 1][1]) % P)
    t1 = xi(*pr[2, 2])
    return [(pr[0, 0][0] + t0[0]) % P, (pr[0, 0][1] + t0[1]) % P,
            (pr[0, 1][0] + pr[1, 0][0] + t1[0]) % P, (pr[0, 1][1] + pr[1, 0][1] + t1[1]) % P,
            (pr[0, 2][0] + pr[1, 1][0] + pr[2, 0][0]) % P, (pr[0, 2][1] + pr[1, 1][1] + pr[2, 0][1]) % P]


def test_e6_tower():
    for s in range(5):
        a, b = rnd(6, s).tolist(), rnd(6, s + 10).tolist()
        got = F.from_mont(oracle.e6_mul(F.to_mont(a), F.to_mont(b))).tolist()
        assert got == _e6_mul_py(a, b)
        inv = oracle.e6_inv(F.to_mont(a))
        one = F.from_mont(oracle.e6_mul(F.to_mont(a), inv)).tolist()
        assert one == [1, 0, 0, 0, 0, 0]


def test_fri_fold_bitreversed_matches_normal_order():
    # fold_bitrev_test.go: fold of bit-reversed evaluations == fold in normal order
    logn = 5
    n = 1 << logn
    coeffs = [rnd(6, 40 + k).tolist() for k in range(n // 2)]  # degree < n/2 E6 polynomial
    w = F.root_of_unity(n)
    alpha = rnd(6, 99).tolist()

    def ev(x, cs):
        acc = [0] * 6
        for c in reversed(cs):
            acc = _e6_mul_py(acc, [x, 0, 0, 0, 0, 0])
            acc = [(acc[i] + c[i]) % P for i in range(6)]
        return acc
    layer = [ev(pow(w, bitrev(r, logn), P), coeffs) for r in range(n)]
    got = F.from_mont(oracle.fri_fold(F.to_mont(np.array(layer, dtype=np.uint32)), F.to_mont(alpha))).tolist()
    # normal order: P_even(x^2) + alpha P_odd(x^2); folded row i is at x_i^2
    even, odd = coeffs[0::2], coeffs[1::2]
    for i in range(n // 2):
        x2 = pow(pow(w, bitrev(i, logn - 1), P), 2, P)
        want = [(a + b) % P for a, b in zip(ev(x2, even), _e6_mul_py(alpha, ev(x2, odd)))]
        assert got[i] == want


@pytest.fixture(scope="module")
def small():
    compiled, wit = plonk.build(2, 1 << 8, seed=11)
    mont = [F.to_mont(w) for w in wit]
    return compiled, wit, mont, oracle.prove(compiled.words, mont, 12)


def test_proof_low_degree_and_vanishing_chunk(small):
    compiled, wit, mont, pb = small
    p = proof.decode(pb)
    assert p.hash_backend == "poseidon2"
    assert len(p.commitments) == 3
    assert all(v == p.final_poly[0] for v in p.final_poly), "FRI final polynomial must be constant"
    for g in p.claimed_values[-1]:
        assert len(g["ext"]) == 4 and g["ext"][3][0] == (0,) * 6, "quotient chunk 3 must vanish (deg Q < 3N)"
    assert len(p.point_samplings) == 12 and all(len(x) == 3 for x in p.point_samplings)


def test_proof_deterministic(small):
    compiled, wit, mont, pb = small
    assert oracle.prove(compiled.words, mont, 12) == pb


def test_tampered_witness_breaks_quotient(small):
    compiled, wit, mont, pb = small
    names = [n for (n, _, _) in compiled.witness_columns]
    bad = [m.copy() for m in mont]
    bad[names.index("O_0")][3] ^= 1
    p = proof.decode(oracle.prove(compiled.words, bad, 12))
    assert any(g["ext"][3][0] != (0,) * 6 for g in p.claimed_values[-1])


def test_broken_copy_constraint_breaks_quotient():
    compiled, wit = plonk.build(1, 1 << 6, seed=13)
    names = [n for (n, _, _) in compiled.witness_columns]
    wit = [w.copy() for w in wit]
    sig = wit[names.index("plonk.S_0_0")]
    sig[[1, 2]] = sig[[2, 1]]
    p = proof.decode(oracle.prove(compiled.words, [F.to_mont(w) for w in wit], 4))
    assert any(g["ext"][3][0] != (0,) * 6 for g in p.claimed_values[-1])


# ---- logup lookups (arguments.Range into a shared 2^8 range table)
@pytest.fixture(scope="module")
def mixed():
    comp, wit = plonk.build_mixed([6, 5, 7, 4], seed=21)
    mont = [F.to_mont(w) for w in wit]
    return comp, wit, mont, oracle.prove(comp.words, mont, 8)


def test_lookup_proof_low_degree_and_balanced_bus(mixed):
    """The FRI final polynomial is constant only if every constraint holds,
    the logup ones included; the exposed totals of a lookup balance to 0
    (the LogupBus the verifier checks, proof/public_inputs.go:55-62)."""
    comp, wit, mont, pb = mixed
    p = proof.decode(pb)
    assert all(v == p.final_poly[0] for v in p.final_poly)
    assert len(p.exposed) == 8  # one logup column per source module and one per lookup in the range module
    tot = [0] * 6
    for ents in p.exposed.values():
        (idx, kind, e), = ents
        assert idx == 0 and kind == 1
        tot = [(a + b) % F.P for a, b in zip(tot, e)]
    assert tot == [0] * 6
    names = sorted(p.exposed)
    assert names[0].startswith("plonk_0.logup_") and names[-1].startswith("range_256.logup_")


def test_lookup_value_outside_table_is_refused(mixed):
    comp, wit, mont, _ = mixed
    i = [c[0] for c in comp.witness_columns].index("RC_2")
    bad = [m.copy() for m in mont]
    bad[i][5] = F.to_mont(np.array([256], dtype=np.uint32))[0]
    with pytest.raises(Exception, match="not in the table"):
        oracle.prove(comp.words, bad, 8)


def test_lookup_proofs_bind_exposed_totals(mixed):
    """A different witness (same range) gives different totals and a
    different transcript."""
    comp, wit, mont, pb = mixed
    i = [c[0] for c in comp.witness_columns].index("RC_0")
    other = [m.copy() for m in mont]
    other[i] = F.to_mont((wit[i].astype(np.uint64) + 1) % 256).astype(np.uint32)
    pb2 = oracle.prove(comp.words, other, 8)
    assert proof.decode(pb2).exposed != proof.decode(pb).exposed
    assert proof.decode(pb2).commitments[1:] != proof.decode(pb).commitments[1:]


# ---- running ratio (board/product.go:72-198)
@pytest.mark.parametrize("permuted", [True, False])
def test_running_ratio_proof(permuted):
    comp, wit, end = plonk.build_with_ratio(64, seed=5, permuted=permuted)
    mont = [F.to_mont(w) for w in wit]
    p = proof.decode(oracle.prove(comp.words, mont, 8))
    assert all(v == p.final_poly[0] for v in p.final_poly)
    (idx, kind, e), = p.exposed[end]
    assert idx == 0 and kind == 1
    assert (tuple(e) == (1, 0, 0, 0, 0, 0)) == permuted

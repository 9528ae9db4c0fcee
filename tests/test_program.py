"""The host program builder mirrors board/arguments: staging order, the
last-round sweep, relation count and degree, generated columns."""
import numpy as np

from loom_b200 import field as F, plonk
from loom_b200.program import KIND_LAGRANGE, KIND_STEP, KIND_WITNESS


def parse(words):
    w = list(map(int, words))
    pos = 0

    def rd():
        nonlocal pos
        pos += 1
        return w[pos - 1]

    def rds():
        n = rd()
        b = b"".join(rd().to_bytes(4, "little") for _ in range((n + 3) // 4))
        return b[:n].decode()
    assert rd() == 0x3150474C
    nr, nm, nc, nn, ns = rd(), rd(), rd(), rd(), rd()
    mods = []
    for _ in range(nm):
        logn = rd(); name = rds(); rels = [rd() for _ in range(rd())]
        mods.append((name, logn, rels))
    cols = [(rds(), rd(), rd(), rd(), rd()) for _ in range(nc)]
    nodes = [(rd(), rd(), rd()) for _ in range(nn)]
    steps = [tuple(rd() for _ in range(6)) for _ in range(ns)]
    staged = [[rd() for _ in range(rd())] for _ in range(nr)]
    assert pos == len(w)
    return nr, mods, cols, nodes, steps, staged


def test_plonk_program_structure():
    compiled, wit = plonk.build(2, 1 << 6, seed=1)
    nr, mods, cols, nodes, steps, staged = parse(compiled.words)
    assert nr == 3
    names = [c[0] for c in cols]
    r0 = [names[i] for i in staged[0]]
    # StageLeaves over Fold(alpha, [A_i, ID_i]) then [A_i, S_i] (arguments/permutation.go:37-127)
    assert r0[:9] == ["L_0", "plonk_0.ID_0_64", "R_0", "plonk_0.ID_1_64", "O_0", "plonk_0.ID_2_64",
                      "plonk.S_0_0", "plonk.S_0_1", "plonk.S_0_2"]
    assert staged[1] == []
    r2 = [names[i] for i in staged[2]]
    assert r2 == sorted(r2) and "gp_1" in r2 and "gp_2" in r2 and "QK_0" in r2
    for name, logn, rels in mods:
        assert len(rels) == 4  # gate, recurrence, two boundary relations
    kinds = {c[0]: c[3] for c in cols}
    assert kinds["gp_1"] == KIND_STEP and kinds["L_0"] == KIND_WITNESS
    assert kinds["plonk_0.Lagrange_0"] == KIND_LAGRANGE
    assert {c[0]: c[2] for c in cols}["gp_1"] == 1  # grand product is E6
    assert len(steps) == 2 and all(s[1] == 2 for s in steps)


def test_witness_satisfies_gates_and_copies():
    n = 1 << 8
    compiled, wit = plonk.build(3, n, seed=2)
    by = {name: w for (name, _, _), w in zip(compiled.witness_columns, wit)}
    for i in range(3):
        assert plonk.check_gates(by, i)
        vals = np.concatenate([by[f"L_{i}"], by[f"R_{i}"], by[f"O_{i}"]]).astype(np.uint64)
        ids = np.concatenate([by[f"plonk_{i}.ID_{k}_{n}"] for k in range(3)])
        sig = np.concatenate([by[f"plonk.S_{i}_{k}"] for k in range(3)])
        pos = {int(v): j for j, v in enumerate(ids)}
        perm = np.array([pos[int(s)] for s in sig])
        assert sorted(perm.tolist()) == list(range(3 * n))
        assert np.array_equal(vals[perm], vals)  # sigma links equal values only


def test_id_support_values():
    from loom_b200.program import id_support
    n = 16
    sup = id_support(3, n)
    w = F.root_of_unity(n)
    assert sup[0].tolist() == [pow(w, j, F.P) for j in range(n)]
    assert sup[2].tolist() == [9 * pow(w, j, F.P) % F.P for j in range(n)]


def test_bus_packs_factors_by_degree():
    """arguments/bus.go:98-137: per module, a running-ratio column takes the
    next denominator and the next numerator in turn while the constraint
    degree stays within 5; bus factors have degree 2, so a column holds one
    receive and two sends (2 + 2 = 4, then 1 + 2 + 2 = 5)."""
    from loom_b200.program import Builder, Module, bus, col
    b = Builder()
    b.add_module(Module("m", 16))
    sends = [([col(f"a{i}"), col(f"b{i}")], "m") for i in range(3)]
    recvs = [([col(f"x{i}"), col(f"y{i}")], "m") for i in range(2)]
    ends = bus(b, [col(f"s{i}") for i in range(3)], [col(f"r{i}") for i in range(2)], sends, recvs)
    steps = b.rounds[2]["steps"]
    assert len(ends) == 2 and b.product_buses == [ends]
    assert [s.end for s in steps] == ends
    assert all(e.startswith("m.busratio_") and e.endswith("_end") for e in ends)
    staged = b.rounds[0]["staged"]
    assert {"a0", "b2", "x1", "y0", "s2", "r1"} <= set(staged)


def _lookup_shaped():
    """rounds_test.go lookupShapedBuilder in spirit: sources s0, s1 of module m
    looked up in t0, t1 of module tab, staged at the fold round."""
    from loom_b200.program import Builder, Module, col, lookup
    b = Builder()
    b.add_module(Module("m", 8))
    b.add_module(Module("tab", 8))
    lookup(b, [(col("s0"), "m"), (col("s1"), "m")], [(col("t0"), "tab"), (col("t1"), "tab")])
    return b


def test_compile_rejects_double_staging():
    """rounds_test.go TestCompileRoundsRejectsDoubleStaging."""
    import pytest
    from loom_b200.program import ROUND_LOG_DERIVATIVE
    b = _lookup_shaped()
    b.stage_columns(ROUND_LOG_DERIVATIVE, "s0")  # already staged at the fold round
    with pytest.raises(ValueError, match="staged twice"):
        b.compile()


def test_staging_in_the_same_round_is_idempotent():
    """rounds_test.go TestStageColumnsSameRoundIsIdempotent."""
    from loom_b200.program import ROUND_FOLD
    a, b = _lookup_shaped(), _lookup_shaped()
    b.stage_columns(ROUND_FOLD, "s0", "t1")
    assert np.array_equal(a.compile().words, b.compile().words)


def test_compile_rejects_unknown_staged_column():
    """rounds_test.go TestCompileRoundsRejectsUnknownColumn."""
    import pytest
    from loom_b200.program import ROUND_FOLD
    b = _lookup_shaped()
    b.stage_columns(ROUND_FOLD, "not_in_any_relation")
    with pytest.raises(ValueError, match="not referenced by any relation"):
        b.compile()

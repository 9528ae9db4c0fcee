"""The phase-level entry points, driven the way the Go prover would drive
them through cgo: the caller keeps the Fiat-Shamir transcript
(loom_b200.transcript, the stand-in for internal/fiat-shamir) and the
library runs each phase — rounds (ExecuteSteps + PCS.Commit), the AIR
quotient, claimed values, DEEP, the FRI levels and rounds, the openings.
The proof that comes out must be byte-identical to lg_prove's (which runs
the same phases with the library's own transcript) and to the oracle's.
The committed-batch handles (lg_commit, lg_session_committed) then evaluate
their polynomials (lg_committed_eval) and open at the query positions
(lg_open_batches) exactly as the proof records."""
import numpy as np
import pytest

import oracle
from loom_b200 import LoomError, _lib, field as F, plonk, proof, transcript

pytestmark = pytest.mark.gpu


def _session_proof(ctx, compiled, mont, q, T=None):
    s = ctx.session(compiled.words, mont, q)
    try:
        return transcript.drive(s, compiled.modules, compiled.n_rounds, q, T), s
    except Exception:
        s.release()
        raise


@pytest.mark.parametrize("batched", [True, False])
def test_session_c1_equals_prove_and_oracle(ctx, batched):
    """The CPU-runnable configuration: 4 plonk modules of 2^12 rows, 200 queries."""
    compiled, wit = plonk.build(4, 1 << 12, seed=0x10AD)
    mont = [F.to_mont(w) for w in wit]
    ctx.set_batched(batched)
    try:
        want = ctx.prove(compiled.words, mont, 200)
        got, s = _session_proof(ctx, compiled, mont, 200)
        s.release()
    finally:
        ctx.set_batched(True)
    assert got == want
    assert got == oracle.prove(compiled.words, mont, 200)


def test_session_mixed_lookup_equals_prove():
    """Uneven modules (several FRI levels entering at different rounds), a
    range lookup with exposed logup totals bound after the round roots."""
    from loom_b200 import Context
    ctx = Context(0)
    compiled, wit = plonk.build_mixed([7, 5, 9, 5], seed=11)
    mont = [F.to_mont(w) for w in wit]
    want = ctx.prove(compiled.words, mont, 24)
    got, s = _session_proof(ctx, compiled, mont, 24)
    assert got == want == oracle.prove(compiled.words, mont, 24)
    assert proof.decode(got).exposed
    ctx.close()  # releases the session first


def test_session_with_setup_root(ctx):
    compiled, wit, setup = plonk.build_with_setup(2, 1 << 7, seed=5)
    wm = [F.to_mont(w) for w in wit]
    sm = [F.to_mont(x) for x in setup]
    ctx.setup(compiled.words, sm)
    want = ctx.prove(compiled.words, wm, 12)
    got, s = _session_proof(ctx, compiled, wm, 12)
    assert s.setup_root() is not None
    s.release()
    assert got == want == oracle.prove(compiled.words, wm, 12, sm)


def test_session_handles_evaluate_and_open_as_the_proof_records(ctx):
    compiled, wit = plonk.build(3, 1 << 8, seed=21)
    mont = [F.to_mont(w) for w in wit]
    T = transcript.Transcript()
    got, s = _session_proof(ctx, compiled, mont, 16, T)
    p = proof.decode(got)
    zeta = T.compute("__zeta")[:6]
    handles = []
    for b, groups in enumerate(p.claimed_values):
        nb = [len(g["base"]) for g in groups]
        ne = [len(g["ext"]) for g in groups]
        h = s.committed(b, nb, ne)
        handles.append(h)
        vals = h.eval(zeta, [0, 1])  # (polys, shifts, 6), Montgomery
        k = 0
        for g in groups:
            for cvs in g["base"] + g["ext"]:
                # the proof holds each polynomial's values at its own shifts:
                # {0} or {0, 1} here
                for si, v in enumerate(cvs):
                    assert F.from_mont(vals[k, si]).tolist() == list(v)
                k += 1
    s.release()  # the handles keep their batches
    # the commitment openings are the proof's last section
    opened = ctx.open_batches(handles, T.positions)
    assert got.endswith(opened)
    for h in handles:
        h.release()


def test_session_refuses_phases_out_of_order(ctx):
    compiled, wit = plonk.build(1, 1 << 6, seed=2)
    mont = [F.to_mont(w) for w in wit]
    s = ctx.session(compiled.words, mont, 4)
    with pytest.raises(LoomError) as e:
        s.commit_round(1)  # round 0's challenge is not known yet
    assert e.value.code == _lib.LG_ERR_INVALID and "challenge@loom_0" in str(e.value)
    with pytest.raises(LoomError):
        s.quotient()
    with pytest.raises(LoomError):
        s.challenge("no_such_challenge", np.zeros(8, np.uint32))
    s.release()
    with pytest.raises(LoomError) as e:
        ctx.session(compiled.words, mont, 4, hash_backend="blake3")
    assert e.value.code == _lib.LG_ERR_UNSUPPORTED


def _e6m(c):
    return F.to_mont(np.array([int(v) % F.P for v in c], dtype=np.uint64))


def _canon(m):
    return [int(x) for x in F.from_mont(m)]


def _eadd(a, b):
    return [(x + y) % F.P for x, y in zip(a, b)]


def _emul(a, b):
    return _canon(oracle.e6_mul(_e6m(a), _e6m(b)))


def _lagrange_eval(rows_c, n, z_c, shift):
    """sum_i L_i(z w^s) P[i], L_i(x) = (x^n - 1)/n w^i/(x - w^i), on canonical
    E6 values (the oracle's E6 product and inverse)."""
    w = F.root_of_unity(n)
    base = lambda x: [x % F.P, 0, 0, 0, 0, 0]  # noqa: E731
    pt = _emul(z_c, base(pow(w, shift, F.P)))
    ptn = base(1)
    for _ in range(n):
        ptn = _emul(ptn, pt)
    common = _emul(_eadd(ptn, base(F.P - 1)), base(pow(n, F.P - 2, F.P)))
    acc = [0] * 6
    for i in range(n):
        wi = pow(w, i, F.P)
        li = _emul(_emul(common, base(wi)), _canon(oracle.e6_inv(_e6m(_eadd(pt, base(F.P - wi))))))
        acc = _eadd(acc, _emul(li, rows_c[i]))
    return acc


def test_commit_handle_root_eval_and_openings(ctx):
    """lg_commit on its own (PCS.Commit of one batch): the root equals the
    root-only entry point's and the oracle's; lg_committed_eval equals direct
    Lagrange evaluation; lg_open_batches returns the oracle's LDE rows around
    each position, a path of the tree's depth and the injected group's rows."""
    rng = np.random.default_rng(99)
    groups = [{"rows": 64, "base": [F.to_mont(rng.integers(0, F.P, 64)) for _ in range(3)],
               "ext": [F.to_mont(rng.integers(0, F.P, 64 * 6))]},
              {"rows": 16, "base": [F.to_mont(rng.integers(0, F.P, 16)) for _ in range(2)]}]
    h = ctx.commit(groups)
    assert np.array_equal(h.root, ctx.commit_root(groups))
    assert np.array_equal(h.root, oracle.commit(groups))  # both Montgomery words
    z = F.to_mont(rng.integers(0, F.P, 6))
    z_c = _canon(z)
    shifts = [0, 3]
    vals = h.eval(z, shifts)
    k = 0
    for g in groups:
        n = g["rows"]
        cols = [(c, False) for c in g.get("base", [])] + [(c, True) for c in g.get("ext", [])]
        for col, ext in cols:
            cc = F.from_mont(np.asarray(col)).reshape(n, 6 if ext else 1)
            rows_c = [list(map(int, r)) + [0] * (6 - cc.shape[1]) for r in cc]
            for si, sh in enumerate(shifts):
                assert _canon(vals[k, si]) == _lagrange_eval(rows_c, n, z_c, sh), (k, sh)
            k += 1
    pos = [0, 5, (1 << 24) - 1, 123457]
    raw = ctx.open_batches([h], pos)
    words = np.frombuffer(raw, dtype=">u4").astype(np.int64)
    big = [F.from_mont(oracle.rs_encode(c, 4 * 64)) for c in groups[0]["base"]]
    big_e = F.from_mont(oracle.rs_encode_e6(groups[0]["ext"][0], 4 * 64)).reshape(-1, 6)
    small = [F.from_mont(oracle.rs_encode(c, 4 * 16)) for c in groups[1]["base"]]
    o = 0
    for s in pos:
        assert words[o] == 1  # one batch
        o += 1
        top_row = (s >> (24 - 8)) & ~1  # 2^8 LDE rows in the larger group
        for r in (top_row, top_row + 1):
            assert words[o] == 3 and words[o + 1:o + 4].tolist() == [int(b[r]) for b in big]
            assert words[o + 4] == 1 and words[o + 5:o + 11].tolist() == big_e[r].tolist()
            o += 11
        assert words[o] == top_row // 2 and words[o + 1] == 7  # leaf index, depth of 2^7 leaves
        o += 2 + 8 * 7
        assert words[o] == 1  # the smaller group's leaf, injected
        o += 1 + 8
        assert words[o] == 1  # and its row pair
        o += 1
        srow = (s >> (24 - 6)) & ~1
        for r in (srow, srow + 1):
            assert words[o] == 2 and words[o + 1:o + 3].tolist() == [int(b[r]) for b in small]
            assert words[o + 3] == 0
            o += 4
    assert o == len(words)
    h.release()


def test_context_budget_and_usage():
    """lg_ctx_create's HBM budget: a prove that needs more than the budget
    fails with LG_ERR_OOM and leaves the context usable; the context's
    high-water mark reports a prove's peak."""
    from loom_b200 import Context
    compiled, wit = plonk.build(2, 1 << 10, seed=4)
    mont = [F.to_mont(w) for w in wit]
    big = Context(0)
    big.mem_usage(reset_peak=True)
    want = big.prove(compiled.words, mont, 8)
    held, peak = big.mem_usage()
    assert peak > 0 and peak >= held
    big.close()
    small = Context(0, hbm_budget=1 << 20)
    with pytest.raises(LoomError) as e:
        small.prove(compiled.words, mont, 8)
    assert e.value.code == _lib.LG_ERR_OOM and "budget" in str(e.value)
    small.close()
    roomy = Context(0, hbm_budget=4 * peak + (256 << 20))
    assert roomy.prove(compiled.words, mont, 8) == want
    roomy.close()

"""The caller-side transcript (loom_b200.transcript), the Python stand-in for
the Go prover's fiat-shamir package that drives the session entry points:
its Poseidon2 permutation and sponge against the oracle's, and the
challenge chaining of internal/fiat-shamir/transcript.go:221-315."""
import numpy as np

import oracle
from loom_b200 import field as F, transcript as T


def test_permutation_equals_oracle():
    rng = np.random.default_rng(7)
    for _ in range(4):
        st = rng.integers(0, F.P, 24).tolist()
        assert T.permute(st) == oracle.p2_permute(np.array(st, dtype=np.uint32)).tolist()


def test_sponge_equals_oracle_for_every_block_shape():
    rng = np.random.default_rng(8)
    for n in (0, 1, 8, 15, 16, 17, 31, 32, 33, 51):
        e = rng.integers(0, F.P, n).tolist()
        want = F.from_mont(oracle.sponge(F.to_mont(np.array(e, dtype=np.uint64)))).tolist()
        assert T.sponge(e) == want, n


def test_string_elements_and_challenge_chain():
    assert T.string_to_elements(T.HASH_TAG, "poseidon2") == [
        T.HASH_TAG, 9, int.from_bytes(b"pos", "little"), int.from_bytes(b"eid", "little"),
        int.from_bytes(b"on2", "little")]
    tr = T.Transcript()
    tr.add("a")
    tr.add("b")
    tr.bind("a", [1, 2, 3])
    tr.bind("b", [4])
    da = tr.canonical("a")
    assert da == T.sponge(T.string_to_elements(T.FSID, "a") + [1, 2, 3])
    assert tr.canonical("b") == T.sponge(T.string_to_elements(T.FSID, "b") + da + [4])
    assert F.from_mont(tr.compute("b")).tolist() == tr.canonical("b")

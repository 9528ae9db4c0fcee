"""Pins of the CPU oracle against the reference's own fixtures and against
independent restatements (no GPU needed)."""
import json
import os
import sys

import numpy as np

import oracle
from loom_b200 import field as F

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "loom_b200", "csrc"))
import gen_constants  # noqa: E402  (the product's constant generator)


def fixture():
    with open(os.path.join(HERE, "golden", "poseidon2_w16_zkc.json")) as f:
        return json.load(f)


def test_width16_round_keys_match_reference_fixture():
    fx = fixture()
    assert oracle.p2_round_keys(16).tolist() == fx["round_keys"]


def test_width16_diagonal_matches_reference_fixture():
    assert oracle.p2_diag(16).tolist() == fixture()["internal_diag"]


def test_product_constants_match_oracle():
    # two independent Keccak restatements (C++ oracle, Python generator)
    keys = gen_constants.round_keys(24)
    flat = [r + [0] * (24 - len(r)) for r in keys]
    assert oracle.p2_round_keys(24).tolist() == flat
    assert oracle.p2_diag(24).tolist() == gen_constants.diag(24)
    assert [r + [0] * (16 - len(r)) for r in gen_constants.round_keys(16)] == fixture()["round_keys"]


def test_keccak_known_answers():
    assert oracle.keccak256(b"").hex() == "c5d2460186f7233c927e7db2dcc703c0e500b653ca82273b7bfad8045d85a470"
    assert oracle.keccak256(b"abc").hex() == "4e03657aea45a94fc7d47ba826c8d667c0d1e6e33a64a036ec44f58fa12d6c45"
    assert gen_constants.keccak256(b"abc") == oracle.keccak256(b"abc")
    long = bytes(range(256)) * 3
    assert gen_constants.keccak256(long) == oracle.keccak256(long)


def test_generator_and_roots():
    p = F.P
    assert pow(3, (p - 1) // 2, p) != 1 and pow(3, (p - 1) // 127, p) != 1
    w = oracle.root_of_unity(1 << 24)
    assert w == 0x6AC49F88
    assert pow(w, 1 << 24, p) == 1 and pow(w, 1 << 23, p) != 1
    for logn in (1, 5, 14, 22):
        assert oracle.root_of_unity(1 << logn) == F.root_of_unity(1 << logn)


def test_width16_diag_structure():
    # M_I = 1.1^T + diag must be invertible and the diagonal distinct
    d = oracle.p2_diag(24).tolist()
    assert len(set(d)) == 24


def _py_perm(state, width):
    """Independent Python restatement of the permutation (round structure of
    recursion/p2_air.go:206-300)."""
    p = F.P
    rk = gen_constants.round_keys(width)
    d = gen_constants.diag(width)
    M4 = [[2, 3, 1, 1], [1, 2, 3, 1], [1, 1, 2, 3], [3, 1, 1, 2]]

    def ext(s):
        out = []
        for c in range(width // 4):
            x = s[4 * c:4 * c + 4]
            out += [sum(M4[r][j] * x[j] for j in range(4)) % p for r in range(4)]
        sums = [sum(out[4 * c + j] for c in range(width // 4)) % p for j in range(4)]
        return [(out[i] + sums[i % 4]) % p for i in range(width)]

    s = ext([x % p for x in state])
    for r in range(27):
        if len(rk[r]) == width:
            s = ext([pow((s[i] + rk[r][i]) % p, 3, p) for i in range(width)])
        else:
            s[0] = pow((s[0] + rk[r][0]) % p, 3, p)
            tot = sum(s) % p
            s = [(tot + d[i] * s[i]) % p for i in range(width)]
    return s


def test_permutation_matches_python_restatement():
    rng = np.random.Generator(np.random.PCG64(5))
    for width in (16, 24):
        for _ in range(3):
            st = rng.integers(0, F.P, width, dtype=np.uint64).tolist()
            assert oracle.p2_permute(st, width).tolist() == _py_perm(st, width)

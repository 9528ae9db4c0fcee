"""Fiat-Shamir transcript on the caller's side of the session entry points.

The Go prover keeps its transcript (internal/fiat-shamir/transcript.go:
124-355) and hands the library only challenges; this module is the same
transcript for Python callers of ``Session``: named challenges declared in
order, each the Poseidon2 sponge (width 24, rate 16, overwrite, no padding,
internal/hash/poseidon2.go:257-393) of the name's elements, the previous
challenge's digest and the values bound to it.  ``drive`` runs a whole prove
through a ``Session`` with it, in the order prover.Prove binds and samples
(prover/prover.go:142-719, internal/fri/open.go:98-285,
internal/fri/fri.go:606-736).

Values cross the C ABI as Montgomery words; the sponge runs on canonical
integers here.  Poseidon2's round keys come from the gnark-crypto parameter
derivation (loom_b200/csrc/gen_constants.py), the linear layers from
recursion/p2_air.go:80-117 and recursion/poseidon2.go:48-90.
"""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import field as F

P = F.P
WIDTH, RATE, DIGEST = 24, 16, 8
FSID, HASH_TAG, SIZE_TAG, FINAL_TAG = 0x46534944, 0x48415348, 0x53495A45, 0x45585450
LOG_N_FRI = 24  # 2^22 largest module x rate 4 (internal/constants/const.go:24-32)
MAX_LOG_MODULE = 22

_RK: Optional[List[List[int]]] = None
_DIAG: Optional[List[int]] = None


def _constants():
    global _RK, _DIAG
    if _RK is None:
        sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc"))
        try:
            import gen_constants as g
        finally:
            sys.path.pop(0)
        _RK, _DIAG = g.round_keys(WIDTH), g.diag(WIDTH)
    return _RK, _DIAG


def _m4(x0, x1, x2, x3):
    # [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] (recursion/p2_air.go:80-104)
    return ((2 * x0 + 3 * x1 + x2 + x3) % P, (x0 + 2 * x1 + 3 * x2 + x3) % P,
            (x0 + x1 + 2 * x2 + 3 * x3) % P, (3 * x0 + x1 + x2 + 2 * x3) % P)


def _external(s: List[int]) -> List[int]:
    y = []
    for c in range(0, WIDTH, 4):
        y.extend(_m4(*s[c:c + 4]))
    sums = [sum(y[j::4]) % P for j in range(4)]
    return [(y[i] + sums[i % 4]) % P for i in range(WIDTH)]


def permute(state: Sequence[int]) -> List[int]:
    """Poseidon2 width 24: M_E, 3 full rounds, 21 partial rounds (lane 0), 3
    full rounds, S-box x^3 (recursion/p2_air.go:206-300); canonical values."""
    rk, d = _constants()
    s = _external([int(x) % P for x in state])
    for r in range(27):
        if r < 3 or r >= 24:
            s = [pow((s[i] + rk[r][i]) % P, 3, P) for i in range(WIDTH)]
            s = _external(s)
        else:
            s[0] = pow((s[0] + rk[r][0]) % P, 3, P)
            tot = sum(s) % P
            s = [(tot + s[i] * d[i]) % P for i in range(WIDTH)]
    return s


def sponge(elems: Sequence[int]) -> List[int]:
    """Digest of canonical elements: blocks of 16 overwrite the state's rate
    part; a partial last block overwrites its own length; no writes: zeros."""
    elems = [int(x) % P for x in elems]
    if not elems:
        return [0] * DIGEST
    state = [0] * WIDTH
    for off in range(0, len(elems), RATE):
        blk = elems[off:off + RATE]
        state[:len(blk)] = blk
        state = permute(state)
    return state[:DIGEST]


def string_to_elements(tag: int, s: str) -> List[int]:
    """tag, byte length, then 3 bytes per element little-endian."""
    b = s.encode()
    out = [tag % P, len(b) % P]
    for i in range(0, len(b), 3):
        out.append(int.from_bytes(b[i:i + 3], "little") % P)
    return out


def _canon(words) -> List[int]:
    return [int(x) for x in F.from_mont(np.asarray(words, dtype=np.uint32).reshape(-1))]


class Transcript:
    """Challenges declared in order; challenge i hashes its name, challenge
    i - 1's digest and its bindings.  Digests come back as Montgomery words,
    the form the session entry points take."""

    def __init__(self):
        self.names: List[str] = []
        self.bindings: Dict[str, List[int]] = {}
        self.values: Dict[str, List[int]] = {}
        self.positions: List[int] = []  # FRI query positions, once drawn

    def add(self, name: str):
        if name in self.bindings:
            raise ValueError("duplicate challenge " + name)
        self.names.append(name)
        self.bindings[name] = []

    def bind(self, name: str, canonical: Sequence[int]):
        if name in self.values:
            raise ValueError("challenge already computed " + name)
        self.bindings[name].extend(int(x) % P for x in canonical)

    def bind_mont(self, name: str, words):
        self.bind(name, _canon(words))

    def compute(self, name: str) -> np.ndarray:
        if name not in self.values:
            i = self.names.index(name)
            elems = string_to_elements(FSID, name)
            if i:
                prev = self.names[i - 1]
                if prev not in self.values:
                    raise ValueError("previous challenge not computed for " + name)
                elems += self.values[prev]
            self.values[name] = sponge(elems + self.bindings[name])
        return F.to_mont(np.array(self.values[name], dtype=np.uint64))

    def canonical(self, name: str) -> List[int]:
        self.compute(name)
        return self.values[name]


def drive(session, modules: Dict[str, int], n_rounds: int, num_queries: int,
          T: Optional[Transcript] = None) -> bytes:
    """The whole prove through `session` (a loom_b200.Session) with a
    transcript (a fresh one unless `T` is given; it keeps every challenge,
    and the query positions in T.positions): `modules` maps module names to
    row counts, as the program declares them.  Returns the proof bytes."""
    T = Transcript() if T is None else T
    coin = [f"challenge@loom_{r}" for r in range(n_rounds)]
    for c in coin:
        T.add(c)
    T.add("__zeta")
    first = coin[0] if coin else "__zeta"
    T.bind(first, string_to_elements(HASH_TAG, "poseidon2"))
    order = sorted(modules)  # layout order: sort.Strings on names (internal/protocol/layout.go:107-114)
    T.bind(first, [SIZE_TAG, len(order)] + [modules[m] for m in order])
    setup_root = session.setup_root()
    if setup_root is not None:
        T.bind_mont(first, setup_root)
    for r in range(n_rounds):
        root, exposed = session.commit_round(r)
        if root is not None:
            T.bind_mont(coin[r], root)
        for e in exposed:  # entry index, then the value (board/logup.go:218-225)
            T.bind(coin[r], [0] + _canon(e))
        session.challenge(coin[r], T.compute(coin[r]))
    root = session.quotient()
    if root is not None:
        T.bind_mont("__zeta", root)
    session.challenge("__zeta", T.compute("__zeta"))
    T.add("alpha_DEEP")
    T.bind_mont("alpha_DEEP", session.claimed_values())
    session.challenge("alpha_DEEP", T.compute("alpha_DEEP"))
    session.deep()
    lroot, n_levels, r0 = session.fri_commit_levels()
    gam = [f"fri_level_{l}_gamma" for l in range(1, n_levels)]
    fold = [f"fri_fold_{j}" for j in range(MAX_LOG_MODULE)]
    query = [f"fri_query_{k}" for k in range(num_queries)]
    for nm in gam + fold + query:
        T.add(nm)
    for i, nm in enumerate(gam):
        if i == 0:
            T.bind_mont(nm, lroot)
        session.challenge(nm, T.compute(nm))
    for j in range(r0):  # rounds before the first layer bind an empty digest
        T.bind(fold[j], [0] * DIGEST)
        T.compute(fold[j])
    T.bind_mont(fold[r0], lroot)
    session.challenge(fold[r0], T.compute(fold[r0]))
    for j in range(r0, MAX_LOG_MODULE):
        nxt = session.fri_fold_round(j)
        if nxt is not None:
            T.bind_mont(fold[j + 1], nxt)
            session.challenge(fold[j + 1], T.compute(fold[j + 1]))
    final = session.fri_final()
    T.bind(query[0], [FINAL_TAG, final.shape[0]] + _canon(final))
    pos = []
    for k in range(num_queries):  # queryIndex (internal/fri/fri.go:1216-1222)
        c = T.canonical(query[k])
        pos.append(((c[0] << 31) ^ c[1]) % (1 << LOG_N_FRI))
        if k + 1 < num_queries:
            T.bind(query[k + 1], c)
    T.positions = pos
    return session.open(pos)

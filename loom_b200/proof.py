"""Decoder of the canonical proof encoding (the mirror of proof.Proof,
proof/proof.go:31-51, fri.OpeningProof internal/fri/pcs.go:131-135 and
fri.Proof internal/fri/fri.go:232-248).

The reference serialises proofs with encoding/gob only to measure their
size, and gob walks Go maps in random order, so there is no canonical byte
format upstream.  This repository defines one, used by the CUDA prover and
checked against the CPU oracle: every integer and every field element is a
4-byte big-endian word, field elements in canonical (non-Montgomery) form,
E6 values as 6 words [B0.A0, B0.A1, B1.A0, B1.A1, B2.A0, B2.A1], digests as
8 words, strings as a length word then the bytes, lists as a count word then
the items, in struct field order.  The exposed values (a Go map) are listed by
name: name, entry count, then per entry its index, its field kind (0 base,
1 extension) and six words (the value as an extension element).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import List


class _R:
    def __init__(self, b: bytes):
        self.b, self.o = b, 0

    def u32(self) -> int:
        v = struct.unpack_from(">I", self.b, self.o)[0]
        self.o += 4
        return v

    def words(self, n: int) -> List[int]:
        v = list(struct.unpack_from(">%dI" % n, self.b, self.o))
        self.o += 4 * n
        return v

    def e6(self):
        return tuple(self.words(6))

    def digest(self):
        return tuple(self.words(8))

    def str(self) -> str:
        n = self.u32()
        s = self.b[self.o:self.o + n].decode()
        self.o += n
        return s


@dataclass
class Path:
    leaf_idx: int
    siblings: list
    injection_leaves: list


@dataclass
class QueryLayer:
    field: int
    row: int
    p: tuple
    q: tuple
    path: Path


@dataclass
class RawRow:
    base: list
    ext: list


@dataclass
class WMerkleProof:
    top: tuple
    path: Path
    injections: list


@dataclass
class Proof:
    hash_backend: str
    exposed: dict              # name -> [(index, field kind, e6)]
    commitments: list
    claimed_values: list       # [batch][group] -> {"base": [[e6]], "ext": [[e6]]}
    levels_root: tuple
    level_queries: list        # [level-1][query] QueryLayer
    fri_roots: list
    final_field: int
    final_poly: list
    fri_queries: list          # [query][layer] QueryLayer
    point_samplings: list      # [query][batch] WMerkleProof
    raw: bytes = field(repr=False, default=b"")


def _path(r: _R) -> Path:
    idx = r.u32()
    sib = [r.digest() for _ in range(r.u32())]
    inj = [r.digest() for _ in range(r.u32())]
    return Path(idx, sib, inj)


def _ql(r: _R) -> QueryLayer:
    f = r.u32()
    row = r.u32()
    if f == 1:
        p, q = r.e6(), r.e6()
    else:
        p, q = (r.u32(),), (r.u32(),)
    return QueryLayer(f, row, p, q, _path(r))


def _row(r: _R) -> RawRow:
    base = r.words(r.u32())
    ext = [r.e6() for _ in range(r.u32())]
    return RawRow(base, ext)


def decode(b: bytes) -> Proof:
    r = _R(b)
    hb = r.str()
    exposed = {}
    for _ in range(r.u32()):
        name = r.str()
        exposed[name] = [(r.u32(), r.u32(), r.e6()) for _ in range(r.u32())]
    commits = [r.digest() for _ in range(r.u32())]
    cvs = []
    for _ in range(r.u32()):
        groups = []
        for _ in range(r.u32()):
            base = [[r.e6() for _ in range(r.u32())] for _ in range(r.u32())]
            ext = [[r.e6() for _ in range(r.u32())] for _ in range(r.u32())]
            groups.append({"base": base, "ext": ext})
        cvs.append(groups)
    levels_root = r.digest()
    lq = [[_ql(r) for _ in range(r.u32())] for _ in range(r.u32())]
    roots = [r.digest() for _ in range(r.u32())]
    ff = r.u32()
    nf = r.u32()
    final = [r.e6() if ff == 1 else (r.u32(),) for _ in range(nf)]
    fq = [[_ql(r) for _ in range(r.u32())] for _ in range(r.u32())]
    if r.u32() != 0:
        raise ValueError("proofs of work are not supported by this decoder")
    ps = []
    for _ in range(r.u32()):
        per = []
        for _ in range(r.u32()):
            top = (_row(r), _row(r))
            path = _path(r)
            inj = [(_row(r), _row(r)) for _ in range(r.u32())]
            per.append(WMerkleProof(top, path, inj))
        ps.append(per)
    if r.o != len(b):
        raise ValueError(f"trailing bytes: {len(b) - r.o}")
    return Proof(hb, exposed, commits, cvs, levels_root, lq, roots, ff, final, fq, ps, b)

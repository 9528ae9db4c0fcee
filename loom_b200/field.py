"""KoalaBear field helpers for the host side (numpy, vectorised).

p = 2^31 - 2^24 + 1.  The device and the C ABI store elements as Montgomery
words with R = 2^32, the in-memory layout of gnark-crypto's
koalabear.Element; these helpers convert canonical values to and from that
form and provide the few exponentiations the column generators need
(board/module.go:229-293).
"""
from __future__ import annotations

import numpy as np

P = 0x7F000001
R_MOD_P = (1 << 32) % P
R_INV = pow(R_MOD_P, P - 2, P)
MULT_GEN = 3  # smallest generator of F_p^*
TWO_ADICITY = 24


def to_mont(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.uint64) % P
    return ((a * R_MOD_P) % P).astype(np.uint32)


def from_mont(m) -> np.ndarray:
    m = np.asarray(m, dtype=np.uint64) % P
    return ((m * R_INV) % P).astype(np.uint32)


def root_of_unity(n: int) -> int:
    """Generator of the subgroup of order n (a power of two <= 2^24)."""
    logn = n.bit_length() - 1
    if n != 1 << logn or logn > TWO_ADICITY:
        raise ValueError(f"no subgroup of order {n}")
    w = pow(MULT_GEN, (P - 1) >> TWO_ADICITY, P)
    return pow(w, 1 << (TWO_ADICITY - logn), P)


def powers(base: int, n: int, start: int = 1) -> np.ndarray:
    """[start, start*base, ..., start*base^(n-1)] mod p, vectorised by doubling."""
    out = np.empty(n, dtype=np.uint64)
    out[0] = start % P
    filled, step = 1, base % P
    while filled < n:
        k = min(filled, n - filled)
        out[filled:filled + k] = (out[:k] * step) % P
        filled += k
        step = step * step % P
    return out.astype(np.uint32)

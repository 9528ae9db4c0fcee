"""Generates p2_constants.h: Poseidon2 width-24 parameters for the device.

gnark-crypto (field/koalabear/poseidon2, v0.22.0, a dependency of loom that
is not vendored) derives round keys from the parameter string
"Poseidon2-koalabear[t=W,rF=6,rP=21,d=3]": h_0 = Keccak-256(seed),
h_i = Keccak-256(h_{i-1}), key_i = big-endian(h_i) mod p; full rounds take W
keys, partial rounds one (call sites: internal/hash/poseidon2.go:51-54).
The internal-layer diagonal follows recursion/poseidon2.go:48-90.

Keys and diagonal are written in Montgomery form (R = 2^32).  Run:
    python loom_b200/csrc/gen_constants.py > loom_b200/csrc/p2_constants.h
"""
import sys

P = 0x7F000001
_RC = [0x0000000000000001, 0x0000000000008082, 0x800000000000808A, 0x8000000080008000,
       0x000000000000808B, 0x0000000080000001, 0x8000000080008081, 0x8000000000008009,
       0x000000000000008A, 0x0000000000000088, 0x0000000080008009, 0x000000008000000A,
       0x000000008000808B, 0x800000000000008B, 0x8000000000008089, 0x8000000000008003,
       0x8000000000008002, 0x8000000000000080, 0x000000000000800A, 0x800000008000000A,
       0x8000000080008081, 0x8000000000008080, 0x0000000080000001, 0x8000000080008008]
_ROT = [[0, 36, 3, 41, 18], [1, 44, 10, 45, 2], [62, 6, 43, 15, 61], [28, 55, 25, 21, 56], [27, 20, 39, 8, 14]]
_M = (1 << 64) - 1


def _rol(x, n):
    return ((x << n) | (x >> (64 - n))) & _M if n else x


def _keccak_f(A):
    for rc in _RC:
        C = [A[x][0] ^ A[x][1] ^ A[x][2] ^ A[x][3] ^ A[x][4] for x in range(5)]
        D = [C[(x - 1) % 5] ^ _rol(C[(x + 1) % 5], 1) for x in range(5)]
        A = [[A[x][y] ^ D[x] for y in range(5)] for x in range(5)]
        B = [[0] * 5 for _ in range(5)]
        for x in range(5):
            for y in range(5):
                B[y][(2 * x + 3 * y) % 5] = _rol(A[x][y], _ROT[x][y])
        A = [[B[x][y] ^ ((~B[(x + 1) % 5][y]) & B[(x + 2) % 5][y]) for y in range(5)] for x in range(5)]
        A[0][0] ^= rc
    return A


def keccak256(msg: bytes) -> bytes:
    """Original Keccak-256 (0x01 padding), from the Keccak specification."""
    rate = 136
    m = bytearray(msg) + b"\x01"
    m += b"\0" * (-len(m) % rate)
    m[-1] |= 0x80
    A = [[0] * 5 for _ in range(5)]
    for off in range(0, len(m), rate):
        for i in range(rate // 8):
            A[i % 5][i // 5] ^= int.from_bytes(m[off + 8 * i:off + 8 * i + 8], "little")
        A = _keccak_f(A)
    return b"".join(A[i % 5][i // 5].to_bytes(8, "little") for i in range(4))


def round_keys(width, rf=6, rp=21):
    h = keccak256(f"Poseidon2-koalabear[t={width},rF={rf},rP={rp},d=3]".encode())
    out = []

    def nxt():
        nonlocal h
        h = keccak256(h)
        return int.from_bytes(h, "big") % P

    for _ in range(rf // 2):
        out.append([nxt() for _ in range(width)])
    for _ in range(rp):
        out.append([nxt()])
    for _ in range(rf // 2):
        out.append([nxt() for _ in range(width)])
    return out


def diag(width):
    pos, negs = {16: ([8, 3, 24], [8, 3, 4, 24]), 24: ([8, 2, 3, 4, 5, 6, 24], [8, 3, 4, 5, 6, 7, 9, 24])}[width]
    ip2 = lambda n: pow(pow(2, n, P), P - 2, P)
    d = [P - 2, 1, 2, ip2(1), 3, 4, P - ip2(1), P - 3, P - 4]
    d += [ip2(n) for n in pos] + [(P - ip2(n)) % P for n in negs]
    return d


def mont(x):
    return (x << 32) % P


def main(out=sys.stdout):
    rk = round_keys(24)
    full = [r for r in rk if len(r) == 24]
    part = [r[0] for r in rk if len(r) == 1]
    w = out.write
    w("// Generated by gen_constants.py: Poseidon2 width 24 (6 full, 21 partial\n")
    w("// rounds, x^3) round keys and internal diagonal, Montgomery form.\n#pragma once\n")
    w("#define LG_P2_FULL_RK_INIT { \\\n")
    for r in full:
        w("  {" + ", ".join("0x%08xu" % mont(x) for x in r) + "}, \\\n")
    w("}\n#define LG_P2_PARTIAL_RK_INIT {" + ", ".join("0x%08xu" % mont(x) for x in part) + "}\n")
    w("#define LG_P2_DIAG_INIT {" + ", ".join("0x%08xu" % mont(x) for x in diag(24)) + "}\n")


if __name__ == "__main__":
    main()

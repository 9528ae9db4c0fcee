"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a C++ restatement of loom's Poseidon2 prove path used to check
the CUDA implementation byte for byte.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline leg may import this module; the product library
(loom_b200) never does.  Build with ``make -C oracle``.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_prove.argtypes = [u32p, ctypes.c_size_t, ctypes.POINTER(u32p), ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_last_proof.argtypes = [ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_verify.argtypes = [u32p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32,
                                    ctypes.c_char_p, u32p, ctypes.c_uint32]
        L.oracle_setup.argtypes = [u32p, ctypes.c_size_t, ctypes.POINTER(u32p), u32p]
        L.oracle_p2_permute.argtypes = [u32p, ctypes.c_int]
        L.oracle_p2_round_keys.argtypes = [ctypes.c_int, u32p]
        L.oracle_p2_diag.argtypes = [ctypes.c_int, u32p]
        L.oracle_keccak256.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint8)]
        L.oracle_root_of_unity.argtypes = [ctypes.c_uint64]
        L.oracle_root_of_unity.restype = ctypes.c_uint32
        L.oracle_rs_encode.argtypes = [u32p, ctypes.c_size_t, ctypes.c_size_t, u32p]
        L.oracle_rs_encode_e6.argtypes = [u32p, ctypes.c_size_t, ctypes.c_size_t, u32p]
        L.oracle_e6_mul.argtypes = [u32p, u32p, u32p]
        L.oracle_e6_inv.argtypes = [u32p, u32p]
        L.oracle_sponge.argtypes = [u32p, ctypes.c_size_t, u32p]
        L.oracle_commit.argtypes = [ctypes.c_uint32, u64p, u32p, u32p, ctypes.POINTER(u32p), u32p, u32p]
        L.oracle_merkle_root.argtypes = [u32p, ctypes.c_size_t, ctypes.c_uint32, u64p, u32p, u32p]
        L.oracle_merkle_root.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(u32p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


class VerifyError(Exception):
    """The oracle's verifier rejected a proof."""


def verify(program_words: np.ndarray, proof: bytes, num_queries: int, logup_buses: Sequence[Sequence[str]] = (),
           product_buses: Sequence[Sequence[str]] = (), setup_root=None) -> None:
    """Checks proof bytes against the program the way loom's verifier does
    (transcript replay, buses, AIR relation at zeta, FRI, Merkle openings,
    DEEP bridge); raises VerifyError with the reason when it rejects.
    `setup_root` (8 canonical words) is the verification key of a program
    with setup columns."""
    L = lib()
    prog = _u32(program_words)
    spec = ";".join(["P:" + ",".join(b) for b in product_buses] + ["L:" + ",".join(b) for b in logup_buses])
    vk = _u32(setup_root if setup_root is not None else np.zeros(8, np.uint32))
    rc = L.oracle_verify(_p(prog), prog.size, bytes(proof), len(proof), num_queries, spec.encode(), _p(vk),
                         0 if setup_root is None else 1)
    if rc != 0:
        raise VerifyError(L.oracle_last_error().decode(errors="replace"))


def setup_root(program_words: np.ndarray, setup_mont: Sequence[np.ndarray]) -> np.ndarray:
    """Root of the setup tree (the verification key, 8 canonical words) of a
    program's setup columns (Montgomery words, descriptor order)."""
    L = lib()
    prog = _u32(program_words)
    cols = [_u32(c) for c in setup_mont]
    arr = (u32p * max(1, len(cols)))(*[_p(c) for c in cols])
    out = np.zeros(8, np.uint32)
    if L.oracle_setup(_p(prog), prog.size, arr, _p(out)) != 0:
        raise RuntimeError("oracle_setup: " + L.oracle_last_error().decode())
    return out


def prove(program_words: np.ndarray, witness_mont: Sequence[np.ndarray], num_queries: int,
          setup_mont: Sequence[np.ndarray] = ()) -> bytes:
    """Proof bytes (canonical encoding) for Montgomery-form witness columns
    (and setup columns, for a program that has them), descriptor order."""
    L = lib()
    prog = _u32(program_words)
    cols = [_u32(c) for c in list(witness_mont) + list(setup_mont)]
    arr = (u32p * max(1, len(cols)))(*[_p(c) for c in cols])
    buf = (ctypes.c_uint8 * (1 << 20))()
    need = ctypes.c_size_t(1 << 20)
    rc = L.oracle_prove(_p(prog), prog.size, arr, num_queries, buf, ctypes.byref(need))
    if rc == 1:  # larger than the first buffer: the oracle kept it
        buf = (ctypes.c_uint8 * need.value)()
        rc = L.oracle_last_proof(buf, ctypes.byref(need))
    if rc == 0:
        return bytes(buf[:need.value])
    raise RuntimeError("oracle_prove: " + L.oracle_last_error().decode())


def p2_permute(state, width: int = 24) -> np.ndarray:
    s = _u32(state).copy()
    lib().oracle_p2_permute(_p(s), width)
    return s


def p2_round_keys(width: int) -> np.ndarray:
    out = np.zeros(27 * width, dtype=np.uint32)
    lib().oracle_p2_round_keys(width, _p(out))
    return out.reshape(27, width)


def p2_diag(width: int) -> np.ndarray:
    out = np.zeros(width, dtype=np.uint32)
    lib().oracle_p2_diag(width, _p(out))
    return out


def keccak256(msg: bytes) -> bytes:
    out = (ctypes.c_uint8 * 32)()
    lib().oracle_keccak256(msg, len(msg), out)
    return bytes(out)


def root_of_unity(n: int) -> int:
    return int(lib().oracle_root_of_unity(n))


def rs_encode(col_mont, big: int) -> np.ndarray:
    c = _u32(col_mont)
    out = np.zeros(big, dtype=np.uint32)
    lib().oracle_rs_encode(_p(c), c.size, big, _p(out))
    return out


def rs_encode_e6(col_mont, big: int) -> np.ndarray:
    c = _u32(col_mont).reshape(-1)
    out = np.zeros(6 * big, dtype=np.uint32)
    lib().oracle_rs_encode_e6(_p(c), c.size // 6, big, _p(out))
    return out


def e6_mul(a, b) -> np.ndarray:
    x, y, o = _u32(a), _u32(b), np.zeros(6, dtype=np.uint32)
    lib().oracle_e6_mul(_p(x), _p(y), _p(o))
    return o


def e6_inv(a) -> np.ndarray:
    x, o = _u32(a), np.zeros(6, dtype=np.uint32)
    lib().oracle_e6_inv(_p(x), _p(o))
    return o


def sponge(elems_mont) -> np.ndarray:
    x, o = _u32(elems_mont), np.zeros(8, dtype=np.uint32)
    lib().oracle_sponge(_p(x), x.size, _p(o))
    return o


def commit(groups: List[dict], with_leaves: bool = False):
    """groups: [{"rows": N, "base": [cols], "ext": [cols (6N words)]}] in
    Montgomery form.  Returns the root (and leaves in sorted group order)."""
    L = lib()
    rows = np.array([g["rows"] for g in groups], dtype=np.uint64)
    nb = np.array([len(g.get("base", [])) for g in groups], dtype=np.uint32)
    ne = np.array([len(g.get("ext", [])) for g in groups], dtype=np.uint32)
    cols = []
    for g in groups:
        cols += [_u32(c) for c in g.get("base", [])] + [_u32(c).reshape(-1) for c in g.get("ext", [])]
    arr = (u32p * max(1, len(cols)))(*[_p(c) for c in cols])
    root = np.zeros(8, dtype=np.uint32)
    n_leaves = int(sum(2 * g["rows"] for g in groups))
    leaves = np.zeros(8 * n_leaves, dtype=np.uint32) if with_leaves else None
    rc = L.oracle_commit(len(groups), rows.ctypes.data_as(u64p), _p(nb), _p(ne), arr, _p(root),
                         _p(leaves) if with_leaves else None)
    if rc != 0:
        raise RuntimeError("oracle_commit: " + L.oracle_last_error().decode())
    return (root, leaves.reshape(-1, 8)) if with_leaves else root


def merkle_root(leaves_mont: np.ndarray, injections: Sequence[np.ndarray] = ()) -> np.ndarray:
    lv = _u32(leaves_mont).reshape(-1)
    widths = np.array([len(_u32(x).reshape(-1)) // 8 for x in injections], dtype=np.uint64)
    inj = np.concatenate([_u32(x).reshape(-1) for x in injections]) if injections else np.zeros(8, dtype=np.uint32)
    root = np.zeros(8, dtype=np.uint32)
    L = lib()
    if L.oracle_merkle_root(_p(lv), lv.size // 8, len(injections), widths.ctypes.data_as(u64p), _p(inj), _p(root)):
        raise ValueError("oracle_merkle_root: " + L.oracle_last_error().decode())
    return root


def fri_fold(layer_mont, alpha_mont) -> np.ndarray:
    L = lib()
    L.oracle_fri_fold.argtypes = [u32p, ctypes.c_size_t, u32p, u32p]
    x = _u32(layer_mont).reshape(-1)
    a = _u32(alpha_mont)
    out = np.zeros(x.size // 2, dtype=np.uint32)
    L.oracle_fri_fold(_p(x), x.size // 6, _p(a), _p(out))
    return out.reshape(-1, 6)


def grand_product(num_mont, den_mont) -> np.ndarray:
    L = lib()
    L.oracle_grand_product.argtypes = [u32p, u32p, ctypes.c_size_t, u32p]
    a, b = _u32(num_mont).reshape(-1), _u32(den_mont).reshape(-1)
    out = np.zeros_like(a)
    L.oracle_grand_product(_p(a), _p(b), a.size // 6, _p(out))
    return out.reshape(-1, 6)


def deep_quotient(lde_mont, alpha_m, z_m, values_m) -> np.ndarray:
    L = lib()
    L.oracle_deep_quotient.argtypes = [u32p, ctypes.c_uint32, ctypes.c_size_t, u32p, u32p, u32p, u32p]
    x = _u32(lde_mont)
    a, z, v = _u32(alpha_m), _u32(z_m), _u32(values_m).reshape(-1)
    out = np.zeros(6 * x.shape[1], dtype=np.uint32)
    L.oracle_deep_quotient(_p(x), x.shape[0], x.shape[1], _p(a), _p(z), _p(v), _p(out))
    return out.reshape(-1, 6)

"""ctypes binding of libloom_gpu.so (the C ABI in include/loom_gpu.h).

The shared library is built in-tree (``python -m loom_b200.build``).  There
is no CPU fallback: when the library or a GPU is missing, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading
import weakref
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libloom_gpu.so")

LG_OK, LG_ERR_INVALID, LG_ERR_CUDA, LG_ERR_OOM, LG_ERR_UNSUPPORTED, LG_ERR_BUFFER = range(6)
EXPORTS = ["lg_ctx_create", "lg_ctx_destroy", "lg_ctx_set_batched", "lg_ctx_set_leaf_mapping", "lg_ctx_set_tuning",
           "lg_ctx_get_tuning", "lg_mem_info", "lg_last_error", "lg_prove", "lg_last_proof", "lg_setup", "lg_verify", "lg_commit_root",
           "lg_rs_encode", "lg_poseidon2_permute", "lg_merkle_root", "lg_fri_fold", "lg_timer_mark",
           "lg_timer_elapsed", "lg_kernel_launches", "lg_jit_kernels", "lg_profile", "lg_profile_report", "lg_grand_product", "lg_grand_product_noalloc", "lg_deep_quotient",
           "lg_ctx_mem_usage", "lg_device_mem_info", "lg_commit", "lg_committed_eval", "lg_open_batches", "lg_session_begin",
           "lg_session_setup_root", "lg_session_challenge", "lg_commit_round", "lg_quotient", "lg_claimed_values",
           "lg_deep", "lg_fri_commit_levels", "lg_fri_fold_round", "lg_fri_final", "lg_open", "lg_session_committed",
           "lg_release"]

u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None
_lock = threading.Lock()


class LoomError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise LoomError(LG_ERR_UNSUPPORTED, f"{LIB_PATH} is not built; run python -m loom_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.lg_ctx_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(vp)]
        L.lg_ctx_mem_usage.argtypes = [vp, u64p, u64p, ctypes.c_int]
        L.lg_device_mem_info.argtypes = [ctypes.c_int, u64p, u64p]
        szp = ctypes.POINTER(ctypes.c_size_t)
        ip = ctypes.POINTER(ctypes.c_int)
        L.lg_commit.argtypes = [vp, ctypes.c_uint32, u64p, u32p, u32p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                ctypes.POINTER(vp), u32p]
        L.lg_committed_eval.argtypes = [vp, vp, u32p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32), u32p]
        L.lg_open_batches.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(vp), u32p, ctypes.c_uint32,
                                      ctypes.POINTER(ctypes.c_uint8), szp]
        L.lg_session_begin.argtypes = [vp, ctypes.c_char_p, u32p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(vp)]
        L.lg_session_setup_root.argtypes = [vp, u32p, ip]
        L.lg_session_challenge.argtypes = [vp, ctypes.c_char_p, u32p]
        L.lg_commit_round.argtypes = [vp, ctypes.c_uint32, u32p, ip, u32p, u32p]
        L.lg_quotient.argtypes = [vp, u32p, ip]
        L.lg_claimed_values.argtypes = [vp, u32p, szp]
        L.lg_deep.argtypes = [vp]
        L.lg_fri_commit_levels.argtypes = [vp, u32p, u32p, u32p]
        L.lg_fri_fold_round.argtypes = [vp, ctypes.c_uint32, u32p, ip]
        L.lg_fri_final.argtypes = [vp, u32p, szp]
        L.lg_open.argtypes = [vp, u32p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint8), szp]
        L.lg_session_committed.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(vp)]
        L.lg_release.argtypes = [vp]
        L.lg_release.restype = None
        L.lg_ctx_destroy.argtypes = [vp]
        L.lg_ctx_destroy.restype = None
        L.lg_ctx_set_batched.argtypes = [vp, ctypes.c_int]
        L.lg_ctx_set_leaf_mapping.argtypes = [vp, ctypes.c_int]
        L.lg_ctx_set_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.c_int64]
        L.lg_ctx_get_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        L.lg_mem_info.argtypes = [vp, u64p, u64p]
        L.lg_last_error.argtypes = [vp]
        L.lg_last_error.restype = ctypes.c_char_p
        L.lg_prove.argtypes = [vp, ctypes.c_char_p, u32p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                               ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_size_t)]
        L.lg_last_proof.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_size_t)]
        L.lg_setup.argtypes = [vp, u32p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int, u32p]
        L.lg_verify.argtypes = [vp, u32p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32, u32p,
                                ctypes.c_char_p]
        L.lg_commit_root.argtypes = [vp, ctypes.c_uint32, u64p, u32p, u32p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, u32p]
        L.lg_rs_encode.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int]
        L.lg_poseidon2_permute.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]
        L.lg_merkle_root.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, u64p, ctypes.c_void_p,
                                     ctypes.c_int, u32p]
        L.lg_fri_fold.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, u32p, ctypes.c_void_p, ctypes.c_int]
        L.lg_deep_quotient.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_int]
        L.lg_grand_product.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int]
        L.lg_grand_product_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                               ctypes.c_void_p]
        L.lg_timer_mark.argtypes = [vp, ctypes.c_uint32]
        L.lg_timer_elapsed.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float)]
        L.lg_kernel_launches.argtypes = []
        L.lg_kernel_launches.restype = ctypes.c_uint64
        L.lg_jit_kernels.argtypes = []
        L.lg_jit_kernels.restype = ctypes.c_uint64
        L.lg_profile.argtypes = [vp, ctypes.c_int]
        L.lg_profile_report.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_size_t)]
        _lib = L
        return L


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """A device context (lg_ctx): one CUDA stream, caches and memory pool."""

    def __init__(self, device: int = 0, tuning: Optional[dict] = None, hbm_budget: int = 0):
        """`tuning`: launch-shape values to apply (see set_tuning), e.g. the
        "params" of loom_b200.autotune.autotune().  `hbm_budget`: device
        bytes this context may hold at once (0: no cap)."""
        self.L = load()
        self.device = device
        self.h = ctypes.c_void_p()
        rc = self.L.lg_ctx_create(device, int(hbm_budget), ctypes.byref(self.h))
        if rc != LG_OK:
            raise LoomError(rc, f"lg_ctx_create failed on device {device}")
        self._proof_cap = 1 << 22
        self._proof_buf = (ctypes.c_uint8 * self._proof_cap)()
        self._handles = weakref.WeakSet()  # sessions and committed batches made on this context
        if tuning:
            self.apply_tuning(tuning)

    def close(self):
        if self.h:
            for hd in list(self._handles):  # handles go before their context
                hd.release()
            self.L.lg_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != LG_OK:
            raise LoomError(rc, self.L.lg_last_error(self.h).decode())

    def set_batched(self, batched: bool):
        """Batched (default): one launch per phase over all groups/modules;
        plain: one launch per group/module."""
        self._check(self.L.lg_ctx_set_batched(self.h, int(batched)))

    def mem_info(self):
        """(free, total) device bytes."""
        f, t = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.L.lg_mem_info(self.h, ctypes.byref(f), ctypes.byref(t)))
        return int(f.value), int(t.value)

    def device_available(self) -> int:
        """Device bytes a new allocation can get now (free memory plus the
        memory pool's unused reserve); waits for no stream."""
        a, t = ctypes.c_uint64(), ctypes.c_uint64()
        rc = self.L.lg_device_mem_info(self.device, ctypes.byref(a), ctypes.byref(t))
        if rc != LG_OK:
            raise LoomError(rc, "lg_device_mem_info failed")
        return int(a.value)

    def mem_usage(self, reset_peak: bool = False):
        """(held, peak) device bytes of this context; reset_peak restarts the
        high-water mark from the bytes held now."""
        h, pk = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.L.lg_ctx_mem_usage(self.h, ctypes.byref(h), ctypes.byref(pk), int(reset_peak)))
        return int(h.value), int(pk.value)

    TUNING_NAMES = ("p2_leaf_min_per_sm", "p2_node_min_per_sm", "p2_inject_min_per_sm", "merkle_tail",
                    "merkle_subtree", "inject_block", "leaf_block", "lde_split", "lde_fwd_threads", "fri_tail_leaves", "quotient_jit",
                    "upload_split")

    def set_tuning(self, name: str, value: int):
        """Launch-shape choice (see include/loom_gpu.h); proofs do not depend on it."""
        self._check(self.L.lg_ctx_set_tuning(self.h, name.encode(), int(value)))

    def get_tuning(self, name: str) -> int:
        v = ctypes.c_int64()
        self._check(self.L.lg_ctx_get_tuning(self.h, name.encode(), ctypes.byref(v)))
        return int(v.value)

    def tuning(self) -> dict:
        return {n: self.get_tuning(n) for n in self.TUNING_NAMES}

    def apply_tuning(self, params: dict):
        for n, v in params.items():
            self.set_tuning(n, v)

    def set_leaf_mapping(self, lanes: int):
        """Poseidon2 leaf hashing: 1 or 6 lanes per permutation, 0 = auto."""
        self._check(self.L.lg_ctx_set_leaf_mapping(self.h, lanes))

    # ------------------------------------------------------------------ prove
    def setup(self, program_words: np.ndarray, setup_cols: Sequence, on_device: bool = False) -> np.ndarray:
        """setup.Setup: precommits the program's setup columns (Montgomery,
        descriptor order; device addresses with on_device=True) on this
        context; returns the root (the verification key, Montgomery words)."""
        prog = _u32(program_words)
        if on_device:
            arr = (ctypes.c_void_p * max(1, len(setup_cols)))(*[int(p) for p in setup_cols])
        else:
            cols = [_u32(c) for c in setup_cols]
            arr = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        root = np.zeros(8, dtype=np.uint32)
        self._check(self.L.lg_setup(self.h, prog.ctypes.data_as(u32p), prog.size, ctypes.cast(arr, ctypes.c_void_p),
                                    int(on_device), root.ctypes.data_as(u32p)))
        return root

    def verify(self, program_words: np.ndarray, proof_bytes: bytes, num_queries: int, logup_buses=(),
               product_buses=(), setup_root=None) -> None:
        """verifier.Verify on the GPU; raises LoomError (code 1, "proof
        rejected: ...") when the proof does not verify.  `setup_root`: the
        verification key (Montgomery words) of a program with setup columns."""
        prog = _u32(program_words)
        spec = ";".join(["P:" + ",".join(b) for b in product_buses] + ["L:" + ",".join(b) for b in logup_buses])
        root = None if setup_root is None else _u32(setup_root)
        self._check(self.L.lg_verify(self.h, prog.ctypes.data_as(u32p), prog.size, bytes(proof_bytes), len(proof_bytes),
                                     num_queries, None if root is None else root.ctypes.data_as(u32p), spec.encode()))

    def prove(self, program_words: np.ndarray, witness: Sequence, num_queries: int, on_device: bool = False,
              hash_backend: str = "poseidon2") -> bytes:
        """prover.Prove with the Poseidon2 backend.  `witness`: Montgomery
        columns in descriptor order — numpy arrays (host) or, with
        on_device=True, integer device addresses (e.g. torch data_ptr())."""
        prog = _u32(program_words)
        if on_device:
            arr = (ctypes.c_void_p * max(1, len(witness)))(*[int(p) for p in witness])
        else:
            cols = [_u32(c) for c in witness]
            arr = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        n = ctypes.c_size_t(self._proof_cap)
        rc = self.L.lg_prove(self.h, hash_backend.encode(), prog.ctypes.data_as(u32p), prog.size, arr, int(on_device),
                             num_queries, self._proof_buf, ctypes.byref(n))
        if rc == LG_ERR_BUFFER:
            self._proof_cap = int(n.value) * 2
            self._proof_buf = (ctypes.c_uint8 * self._proof_cap)()
            n = ctypes.c_size_t(self._proof_cap)
            rc = self.L.lg_last_proof(self.h, self._proof_buf, ctypes.byref(n))
        self._check(rc)
        return bytes(memoryview(self._proof_buf)[:n.value])

    def prove_into(self, out, program_words: np.ndarray, witness: Sequence, num_queries: int,
                   on_device: bool = False, hash_backend: str = "poseidon2") -> int:
        """prove() writing the proof straight into `out` (a writable buffer:
        bytearray, numpy uint8 array, ...), without the copy into a new bytes
        object.  Returns the proof length; raises LoomError (LG_ERR_BUFFER,
        needed size in the message) when `out` is too small."""
        prog = _u32(program_words)
        if on_device:
            arr = (ctypes.c_void_p * max(1, len(witness)))(*[int(p) for p in witness])
        else:
            cols = [_u32(c) for c in witness]
            arr = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        mv = memoryview(out).cast("B")
        if mv.readonly:
            raise TypeError("out must be writable")
        buf = (ctypes.c_uint8 * len(mv)).from_buffer(mv)
        n = ctypes.c_size_t(len(mv))
        rc = self.L.lg_prove(self.h, hash_backend.encode(), prog.ctypes.data_as(u32p), prog.size, arr, int(on_device),
                             num_queries, buf, ctypes.byref(n))
        if rc == LG_ERR_BUFFER:
            raise LoomError(rc, f"output buffer of {len(mv)} bytes is too small: the proof needs {n.value}")
        self._check(rc)
        return int(n.value)

    # ------------------------------------------------------------------ measurement
    def mark(self, slot: int):
        self._check(self.L.lg_timer_mark(self.h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = ctypes.c_float()
        self._check(self.L.lg_timer_elapsed(self.h, a, b, ctypes.byref(ms)))
        return float(ms.value)

    def kernel_launches(self) -> int:
        return int(self.L.lg_kernel_launches())

    def profile(self, enable: bool):
        self._check(self.L.lg_profile(self.h, int(enable)))

    def profile_report(self) -> dict:
        import json
        n = ctypes.c_size_t(1 << 16)
        buf = ctypes.create_string_buffer(n.value)
        rc = self.L.lg_profile_report(self.h, buf, ctypes.byref(n))
        if rc == LG_ERR_BUFFER:
            buf = ctypes.create_string_buffer(n.value)
            rc = self.L.lg_profile_report(self.h, buf, ctypes.byref(n))
        self._check(rc)
        return json.loads(buf.value.decode())

    # ------------------------------------------------------------------ phase entry points
    def commit_root(self, groups: List[dict]) -> np.ndarray:
        rows = np.array([g["rows"] for g in groups], dtype=np.uint64)
        nb = np.array([len(g.get("base", [])) for g in groups], dtype=np.uint32)
        ne = np.array([len(g.get("ext", [])) for g in groups], dtype=np.uint32)
        cols = []
        for g in groups:
            cols += [_u32(c) for c in g.get("base", [])] + [_u32(c).reshape(-1) for c in g.get("ext", [])]
        arr = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        root = np.zeros(8, dtype=np.uint32)
        self._check(self.L.lg_commit_root(self.h, len(groups), rows.ctypes.data_as(u64p), nb.ctypes.data_as(u32p),
                                          ne.ctypes.data_as(u32p), arr, 0, root.ctypes.data_as(u32p)))
        return root

    def _batch_args(self, groups: List[dict]):
        rows = np.array([g["rows"] for g in groups], dtype=np.uint64)
        nb = np.array([len(g.get("base", [])) for g in groups], dtype=np.uint32)
        ne = np.array([len(g.get("ext", [])) for g in groups], dtype=np.uint32)
        cols = []
        for g in groups:
            cols += [_u32(c) for c in g.get("base", [])] + [_u32(c).reshape(-1) for c in g.get("ext", [])]
        arr = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        return rows, nb, ne, cols, arr

    def commit(self, groups: List[dict]) -> "Committed":
        """PCS.Commit keeping the batch on the device: groups of
        {"rows": N, "base": [N words], "ext": [N x 6 words]} (Montgomery)."""
        rows, nb, ne, cols, arr = self._batch_args(groups)
        root = np.zeros(8, dtype=np.uint32)
        h = ctypes.c_void_p()
        self._check(self.L.lg_commit(self.h, len(groups), rows.ctypes.data_as(u64p), nb.ctypes.data_as(u32p),
                                     ne.ctypes.data_as(u32p), arr, 0, ctypes.byref(h), root.ctypes.data_as(u32p)))
        return Committed(self, h, root, [int(x) for x in nb], [int(x) for x in ne])

    def open_batches(self, batches: Sequence["Committed"], positions: Sequence[int]) -> bytes:
        """Openings of committed batches at FRI positions, in the proof's
        encoding (openCommittedAt for every position)."""
        hs = (ctypes.c_void_p * len(batches))(*[b.h.value for b in batches])
        pos = _u32(positions)
        n = ctypes.c_size_t(0)
        rc = self.L.lg_open_batches(self.h, len(batches), hs, pos.ctypes.data_as(u32p), pos.size, None, ctypes.byref(n))
        if rc != LG_ERR_BUFFER:
            self._check(rc)
        buf = (ctypes.c_uint8 * max(1, n.value))()
        self._check(self.L.lg_open_batches(self.h, len(batches), hs, pos.ctypes.data_as(u32p), pos.size, buf,
                                           ctypes.byref(n)))
        return bytes(memoryview(buf)[:n.value])

    def session(self, program_words: np.ndarray, witness: Sequence, num_queries: int, on_device: bool = False,
                hash_backend: str = "poseidon2") -> "Session":
        """A prove driven phase by phase with the caller's transcript."""
        return Session(self, program_words, witness, num_queries, on_device, hash_backend)

    def rs_encode(self, cols: np.ndarray) -> np.ndarray:
        c = _u32(cols)
        if c.ndim == 1:
            c = c[None, :]
        out = np.zeros((c.shape[0], 4 * c.shape[1]), dtype=np.uint32)
        self._check(self.L.lg_rs_encode(self.h, _ptr(c), c.shape[1], c.shape[0], _ptr(out), 0))
        return out

    def poseidon2_permute(self, states: np.ndarray) -> np.ndarray:
        s = _u32(states).reshape(-1, 24).copy()
        self._check(self.L.lg_poseidon2_permute(self.h, _ptr(s), s.shape[0], 0))
        return s

    def merkle_root(self, leaves: np.ndarray, injections: Sequence[np.ndarray] = ()) -> np.ndarray:
        lv = _u32(leaves).reshape(-1, 8)
        widths = np.array([_u32(x).reshape(-1, 8).shape[0] for x in injections], dtype=np.uint64)
        inj = np.concatenate([_u32(x).reshape(-1) for x in injections]) if injections else np.zeros(8, dtype=np.uint32)
        root = np.zeros(8, dtype=np.uint32)
        self._check(self.L.lg_merkle_root(self.h, _ptr(lv), lv.shape[0], len(injections), widths.ctypes.data_as(u64p),
                                          _ptr(inj), 0, root.ctypes.data_as(u32p)))
        return root

    def deep_quotient(self, lde: np.ndarray, alpha, z, values) -> np.ndarray:
        """Single-point DEEP quotient over base LDE columns (rows bit-reversed)."""
        x = _u32(lde)
        a, zz, v = _u32(alpha), _u32(z), _u32(values).reshape(-1)
        out = np.zeros((x.shape[1], 6), dtype=np.uint32)
        self._check(self.L.lg_deep_quotient(self.h, _ptr(x), x.shape[0], x.shape[1], a.ctypes.data_as(u32p),
                                            zz.ctypes.data_as(u32p), _ptr(v), _ptr(out), 0))
        return out

    def grand_product(self, num: np.ndarray, den: np.ndarray) -> np.ndarray:
        a, b = _u32(num).reshape(-1, 6), _u32(den).reshape(-1, 6)
        out = np.zeros_like(a)
        self._check(self.L.lg_grand_product(self.h, _ptr(a), _ptr(b), a.shape[0], _ptr(out), 0))
        return out

    def fri_fold(self, layer: np.ndarray, alpha) -> np.ndarray:
        x = _u32(layer).reshape(-1, 6)
        a = _u32(alpha)
        out = np.zeros((x.shape[0] // 2, 6), dtype=np.uint32)
        self._check(self.L.lg_fri_fold(self.h, _ptr(x), x.shape[0], a.ctypes.data_as(u32p), _ptr(out), 0))
        return out


class Committed:
    """A committed batch on the device (lg_committed)."""

    def __init__(self, ctx: Context, h, root: np.ndarray, nb: List[int], ne: List[int]):
        self.ctx, self.h, self.root, self.nb, self.ne = ctx, h, root, nb, ne
        ctx._handles.add(self)

    def eval(self, zeta, shifts: Sequence[int]) -> np.ndarray:
        """Values at zeta w^s of every polynomial (group by group, base then
        ext), each at every shift: (polys, shifts, 6) Montgomery words."""
        z = _u32(zeta)
        sh = np.ascontiguousarray(shifts, dtype=np.int32)
        npoly = sum(self.nb) + sum(self.ne)
        out = np.zeros((npoly, len(sh), 6), dtype=np.uint32)
        self.ctx._check(self.ctx.L.lg_committed_eval(self.ctx.h, self.h, z.ctypes.data_as(u32p), len(sh),
                                                     sh.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                     out.ctypes.data_as(u32p)))
        return out

    def release(self):
        if self.h and self.h.value:
            self.ctx.L.lg_release(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Session:
    """One prove driven phase by phase (lg_session_*): the caller keeps the
    Fiat-Shamir transcript and hands each challenge in by name."""

    def __init__(self, ctx: Context, program_words, witness, num_queries: int, on_device: bool, hash_backend: str):
        self.ctx, self.L = ctx, ctx.L
        prog = _u32(program_words)
        if on_device:
            self._arr = (ctypes.c_void_p * max(1, len(witness)))(*[int(p) for p in witness])
        else:
            self._cols = [_u32(c) for c in witness]
            self._arr = (ctypes.c_void_p * max(1, len(self._cols)))(*[c.ctypes.data for c in self._cols])
        self.h = ctypes.c_void_p()
        ctx._check(self.L.lg_session_begin(ctx.h, hash_backend.encode(), prog.ctypes.data_as(u32p), prog.size,
                                           self._arr, int(on_device), num_queries, ctypes.byref(self.h)))
        ctx._handles.add(self)

    def _ck(self, rc):
        self.ctx._check(rc)

    def setup_root(self):
        root = np.zeros(8, dtype=np.uint32)
        has = ctypes.c_int()
        self._ck(self.L.lg_session_setup_root(self.h, root.ctypes.data_as(u32p), ctypes.byref(has)))
        return root if has.value else None

    def challenge(self, name: str, digest) -> None:
        d = _u32(digest)
        assert d.size == 8
        self._ck(self.L.lg_session_challenge(self.h, name.encode(), d.ctypes.data_as(u32p)))

    def commit_round(self, r: int):
        """(root or None, exposed values as an (n, 6) array)."""
        root = np.zeros(8, dtype=np.uint32)
        com = ctypes.c_int()
        cap = 4096
        ex = np.zeros((cap, 6), dtype=np.uint32)
        n = ctypes.c_uint32(cap)
        self._ck(self.L.lg_commit_round(self.h, r, root.ctypes.data_as(u32p), ctypes.byref(com),
                                        ex.ctypes.data_as(u32p), ctypes.byref(n)))
        return (root if com.value else None), ex[:n.value].copy()

    def quotient(self):
        root = np.zeros(8, dtype=np.uint32)
        com = ctypes.c_int()
        self._ck(self.L.lg_quotient(self.h, root.ctypes.data_as(u32p), ctypes.byref(com)))
        return root if com.value else None

    def _values(self, fn) -> np.ndarray:
        n = ctypes.c_size_t(0)
        rc = fn(None, ctypes.byref(n))
        if rc != LG_ERR_BUFFER:
            self._ck(rc)
        out = np.zeros((max(1, n.value), 6), dtype=np.uint32)
        self._ck(fn(out.ctypes.data_as(u32p), ctypes.byref(n)))
        return out[:n.value]

    def claimed_values(self) -> np.ndarray:
        return self._values(lambda p, n: self.L.lg_claimed_values(self.h, p, n))

    def deep(self):
        self._ck(self.L.lg_deep(self.h))

    def fri_commit_levels(self):
        """(levels root, level count, first round with a layer)."""
        root = np.zeros(8, dtype=np.uint32)
        nl, r0 = ctypes.c_uint32(), ctypes.c_uint32()
        self._ck(self.L.lg_fri_commit_levels(self.h, root.ctypes.data_as(u32p), ctypes.byref(nl), ctypes.byref(r0)))
        return root, int(nl.value), int(r0.value)

    def fri_fold_round(self, j: int):
        root = np.zeros(8, dtype=np.uint32)
        com = ctypes.c_int()
        self._ck(self.L.lg_fri_fold_round(self.h, j, root.ctypes.data_as(u32p), ctypes.byref(com)))
        return root if com.value else None

    def fri_final(self) -> np.ndarray:
        return self._values(lambda p, n: self.L.lg_fri_final(self.h, p, n))

    def open(self, positions: Sequence[int]) -> bytes:
        pos = _u32(positions)
        n = ctypes.c_size_t(0)
        rc = self.L.lg_open(self.h, pos.ctypes.data_as(u32p), pos.size, None, ctypes.byref(n))
        if rc == LG_ERR_BUFFER:
            buf = (ctypes.c_uint8 * n.value)()
            self._ck(self.L.lg_last_proof(self.ctx.h, buf, ctypes.byref(n)))
            return bytes(memoryview(buf)[:n.value])
        self._ck(rc)
        return b""

    def committed(self, index: int, nb: Sequence[int] = (), ne: Sequence[int] = ()) -> Committed:
        """Handle to committed batch `index` (layout order); nb / ne: its
        groups' polynomial counts, for Committed.eval's output shape."""
        h = ctypes.c_void_p()
        self._ck(self.L.lg_session_committed(self.h, index, ctypes.byref(h)))
        return Committed(self.ctx, h, None, list(nb), list(ne))

    def release(self):
        if self.h and self.h.value:
            self.L.lg_release(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

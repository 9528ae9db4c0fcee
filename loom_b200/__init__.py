"""loom_b200 — B200-native (sm_100a) prove phase of loom's Poseidon2 backend.

Host side: ``program`` (board-style program builder), ``plonk`` (seeded
synthetic workloads), ``proof`` (canonical proof decoder) and ``Context``
(ctypes binding of the CUDA library's C ABI, include/loom_gpu.h).
"""
from ._lib import Context, LoomError, load  # noqa: F401
from . import field, program, plonk, proof  # noqa: F401

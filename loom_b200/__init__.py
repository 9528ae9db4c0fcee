"""loom_b200 — B200-native (sm_100a) prove phase of loom's Poseidon2 backend.

Host side: ``program`` (board-style program builder), ``plonk`` (seeded
synthetic workloads), ``proof`` (canonical proof decoder), ``Context`` (ctypes binding of the CUDA
library's C ABI, include/loom_gpu.h), ``Session`` and ``Committed`` (its
phase-level entry points) and ``transcript`` (the caller-side Fiat-Shamir
transcript that drives a ``Session``).
"""
from ._lib import Committed, Context, LoomError, Session, load  # noqa: F401
from . import field, program, plonk, proof, transcript  # noqa: F401

"""The C ABI library loads and exports every symbol include/loom_gpu.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from loom_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "loom_gpu.h")).read()
    return sorted(set(re.findall(r"\b(lg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_expected_symbols():
    assert set(_lib.EXPORTS) <= set(declared())


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for sym in declared():
        assert hasattr(lib, sym), sym


def test_oracle_not_linked_into_product():
    so = open(_lib.LIB_PATH, "rb").read()
    assert b"oracle_prove" not in so and b"liboracle" not in so

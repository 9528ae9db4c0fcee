"""The host-side Poseidon2 of the transcript (loom_b200/csrc/p2_host.cpp,
vectorised with AVX2 where the CPU has it) against the oracle permutation.
Built here with g++ into a temporary library; no GPU needed."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from loom_b200 import field as F

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = r'''
#include "poseidon2.cuh"
extern "C" void host_permute(uint32_t* states, unsigned long n) {
  for (unsigned long i = 0; i < n; i++) lg::p2_permute_host(states + 24 * i);
}
extern "C" void scalar_permute(uint32_t* states, unsigned long n) {
  for (unsigned long i = 0; i < n; i++) lg::p2_permute(states + 24 * i);
}
extern "C" void level_permute(uint32_t* states, unsigned long n, int level) {
  for (unsigned long i = 0; i < n; i++) lg::p2_permute_host_at(states + 24 * i, level);
}
extern "C" int simd_level() { return lg::p2_host_simd_level(); }
'''


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("p2host")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    out = d / "libp2host.so"
    csrc = os.path.join(ROOT, "loom_b200", "csrc")
    subprocess.run([gxx, "-std=c++17", "-O2", "-w", "-shared", "-fPIC", "-I", csrc, str(src),
                    os.path.join(csrc, "p2_host.cpp"), "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    for f in (L.host_permute, L.scalar_permute):
        f.argtypes = [ctypes.c_void_p, ctypes.c_ulong]
    L.level_permute.argtypes = [ctypes.c_void_p, ctypes.c_ulong, ctypes.c_int]
    return L


def test_host_permutation_matches_oracle(lib):
    rng = np.random.Generator(np.random.PCG64(24))
    canon = rng.integers(0, F.P, (300, 24), dtype=np.uint64).astype(np.uint32)
    canon[0] = 0
    canon[1] = F.P - 1
    canon[2] = np.arange(24) % 2
    for name in ("host_permute", "scalar_permute"):
        st = np.ascontiguousarray(F.to_mont(canon))
        getattr(lib, name)(st.ctypes.data, st.shape[0])
        got = F.from_mont(st)
        for i in range(canon.shape[0]):
            assert np.array_equal(got[i], oracle.p2_permute(canon[i], 24)), (name, i)


def test_every_vector_width_matches_oracle(lib):
    """Each width this CPU has (AVX-512 and AVX2 where present, scalar always)
    gives the oracle's permutation."""
    rng = np.random.Generator(np.random.PCG64(25))
    canon = rng.integers(0, F.P, (200, 24), dtype=np.uint64).astype(np.uint32)
    canon[0] = F.P - 1
    for level in range(lib.simd_level() + 1):
        st = np.ascontiguousarray(F.to_mont(canon))
        lib.level_permute(st.ctypes.data, st.shape[0], level)
        got = F.from_mont(st)
        for i in range(canon.shape[0]):
            assert np.array_equal(got[i], oracle.p2_permute(canon[i], 24)), (level, i)

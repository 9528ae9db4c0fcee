"""The library's host Fiat-Shamir transcript (loom_b200/csrc/host.cuh
Transcript, with the vectorised permutation of p2_host.cpp) against the
oracle: challenge = H(FSID-tagged name || previous challenge || bindings)
(internal/fiat-shamir/transcript.go:285-315).  The chains mirror the prove's
two long host stretches: alpha_DEEP over many claimed values, then the query
challenges, each binding the one before.  Built here with nvcc into a
temporary library and run on the host only; no GPU needed."""
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
#include "host.cuh"
extern "C" int chain(const uint32_t* binds, unsigned n_binds, unsigned n_queries, uint32_t* out) {
  try {
    lg::Transcript fs;
    fs.add("alpha_DEEP");
    for (unsigned k = 0; k < n_queries; k++) fs.add("fri_query_" + std::to_string(k));
    const size_t ia = fs.at("alpha_DEEP");
    for (unsigned i = 0; i + 6 <= n_binds; i += 6) fs.bind_at(ia, binds + i, 6);
    const lg::Digest a = fs.compute("alpha_DEEP");
    for (int w = 0; w < 8; w++) out[w] = a.v[w];
    const size_t q0 = fs.at("fri_query_0");
    fs.bind_at(q0, a.v, 8);
    for (unsigned k = 0; k < n_queries; k++) {
      const lg::Digest ch = fs.compute_at(q0 + k);
      for (int w = 0; w < 8; w++) out[8 * (k + 1) + w] = ch.v[w];
      if (k + 1 < n_queries) fs.bind_at(q0 + k + 1, ch.v, 8);
    }
    return 0;
  } catch (...) {
    return 1;
  }
}
'''

FSID = 0x46534944


def name_elements(s: str) -> list:
    """string_to_elements (internal/hash/hash.go:39-58), canonical."""
    b = s.encode()
    out = [FSID % F.P, len(b) % F.P]
    for i in range(0, len(b), 3):
        out.append(int.from_bytes(b[i:i + 3], "little") % F.P)
    return out


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("transcript")
    src = d / "shim.cu"
    src.write_text(SHIM)
    out = d / "libtranscript.so"
    csrc = os.path.join(ROOT, "loom_b200", "csrc")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-w", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                    "-fPIC", "-shared", "-I", csrc, str(src), os.path.join(csrc, "p2_host.cpp"), "-o", str(out)],
                   check=True)
    L = ctypes.CDLL(str(out))
    L.chain.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]
    return L


@pytest.mark.parametrize("n_values,n_queries", [(0, 1), (1, 3), (37, 20), (800, 200)])
def test_transcript_chains_match_oracle(lib, n_values, n_queries):
    rng = np.random.Generator(np.random.PCG64(n_values * 1000 + n_queries))
    canon = rng.integers(0, F.P, 6 * n_values, dtype=np.uint64).astype(np.uint32)
    binds = np.ascontiguousarray(F.to_mont(canon), dtype=np.uint32)
    out = np.zeros(8 * (n_queries + 1), dtype=np.uint32)
    assert lib.chain(binds.ctypes.data, binds.size, n_queries, out.ctypes.data) == 0
    # alpha_DEEP: the first challenge, no previous one
    want = oracle.sponge(np.concatenate([F.to_mont(np.array(name_elements("alpha_DEEP"), dtype=np.uint32)), binds]))
    assert np.array_equal(out[:8], want)
    prev = out[:8]
    for k in range(n_queries):
        name = F.to_mont(np.array(name_elements(f"fri_query_{k}"), dtype=np.uint32))
        bound = out[:8] if k == 0 else out[8 * k:8 * k + 8]
        want = oracle.sponge(np.concatenate([name, prev, bound]))
        got = out[8 * (k + 1):8 * (k + 2)]
        assert np.array_equal(got, want), k
        prev = got

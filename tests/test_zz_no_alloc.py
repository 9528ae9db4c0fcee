"""lg_grand_product_noalloc: the grand product for callers that cannot call
cudaMalloc (a caching allocator owns the device memory, a memory-capped
sandbox, a request path that must not allocate).  They bring device buffers
for inputs and output; the entry point's only scratch is a fixed device
array inside the library.  Its output must equal the allocating entry point
lg_grand_product's, bit for bit (integer arithmetic: the same bar as every
other parity test here), on consecutive calls that reuse that array.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from loom_b200 import Context, _lib, field as F

pytestmark = pytest.mark.gpu


def rnd(shape, seed):
    return np.random.Generator(np.random.PCG64(seed)).integers(0, F.P, shape, dtype=np.uint64).astype(np.uint32)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to("cuda:0")


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    import torch
    L = _lib.load()
    ctx = Context(0)
    stream = torch.cuda.Stream(device=0)
    # two calls in a row; the second covers fewer scan tiles than the first
    for call, n in enumerate([5000, 3001]):
        num = F.to_mont(rnd((n, 6), 10 + call))
        den = F.to_mont(rnd((n, 6), 20 + call))
        want = ctx.grand_product(num, den)
        dn, dd = _dev(torch, num), _dev(torch, den)
        out = torch.zeros_like(dn)
        torch.cuda.synchronize()
        rc = L.lg_grand_product_noalloc(ctypes.c_void_p(dn.data_ptr()), ctypes.c_void_p(dd.data_ptr()), n,
                                        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == _lib.LG_OK
        stream.synchronize()
        got = out.cpu().numpy().view(np.uint32).reshape(n, 6)
        assert np.array_equal(got, want), f"call {call}"
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    L = _lib.load()
    buf = torch.zeros(6 * 16, dtype=torch.int32, device="cuda:0")
    p = ctypes.c_void_p(buf.data_ptr())
    assert L.lg_grand_product_noalloc(p, p, (1 << 22) + 1, p, None) == _lib.LG_ERR_UNSUPPORTED
    assert L.lg_grand_product_noalloc(p, p, 0, p, None) == _lib.LG_ERR_INVALID

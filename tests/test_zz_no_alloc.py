"""lg_grand_product_noalloc: the grand product for callers that cannot call
cudaMalloc (a caching allocator owns the device memory, a memory-capped
sandbox, a request path that must not allocate).  They bring device buffers
for inputs and output; the entry point's only scratch is a fixed device
array inside the library.  Its output must equal the allocating entry point
lg_grand_product's, bit for bit (integer arithmetic: the same bar as every
other parity test here), on consecutive calls that reuse that array —
including a call at the array's full capacity (2^22 rows: 2048 scan tiles
fill both halves of it) and one whose last tile holds a single row.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from loom_b200 import Context, _lib, field as F

pytestmark = pytest.mark.gpu

TILE = 2048  # rows per scan tile of the entry point


def rnd(shape, seed):
    return np.random.Generator(np.random.PCG64(seed)).integers(0, F.P, shape, dtype=np.uint64).astype(np.uint32)


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to("cuda:0")


def _call(L, torch, dn, dd, n, out, stream):
    return L.lg_grand_product_noalloc(ctypes.c_void_p(dn.data_ptr()), ctypes.c_void_p(dd.data_ptr()), n,
                                      ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    import torch
    L = _lib.load()
    ctx = Context(0)
    stream = torch.cuda.Stream(device=0)
    # calls in a row: fewer tiles than the call before, then the full
    # capacity, then a last tile of one row
    for call, n in enumerate([5000, 3001, 1 << 22, 3 * TILE + 1]):
        num = F.to_mont(rnd((n, 6), 10 + call))
        den = F.to_mont(rnd((n, 6), 20 + call))
        want = ctx.grand_product(num, den)
        dn, dd = _dev(torch, num), _dev(torch, den)
        out = torch.zeros_like(dn)
        torch.cuda.synchronize()
        launches = L.lg_kernel_launches()
        assert _call(L, torch, dn, dd, n, out, stream) == _lib.LG_OK
        stream.synchronize()
        assert L.lg_kernel_launches() - launches == 4
        got = out.cpu().numpy().view(np.uint32).reshape(n, 6)
        assert np.array_equal(got, want), f"call {call} (n = {n})"
    ctx.close()


def test_noalloc_leaves_free_device_memory_unchanged():
    import torch
    L = _lib.load()
    stream = torch.cuda.Stream(device=0)
    n = 5 * TILE + 7
    dn = _dev(torch, F.to_mont(rnd((n, 6), 31)))
    dd = _dev(torch, F.to_mont(rnd((n, 6), 32)))
    out = torch.zeros_like(dn)
    assert _call(L, torch, dn, dd, n, out, stream) == _lib.LG_OK  # warm: module load, symbol lookup
    stream.synchronize()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        assert _call(L, torch, dn, dd, n, out, stream) == _lib.LG_OK
    stream.synchronize()
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    L = _lib.load()
    buf = torch.zeros(6 * 16, dtype=torch.int32, device="cuda:0")
    p = ctypes.c_void_p(buf.data_ptr())
    assert L.lg_grand_product_noalloc(p, p, (1 << 22) + 1, p, None) == _lib.LG_ERR_UNSUPPORTED
    assert L.lg_grand_product_noalloc(p, p, 0, p, None) == _lib.LG_ERR_INVALID

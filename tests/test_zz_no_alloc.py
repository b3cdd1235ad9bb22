"""The allocation-free prefix sum (slosh_prefix_sum_noalloc) against the
context-based slosh_prefix_sum, through the C ABI.

The allocation-free entry point serves callers that cannot allocate device
memory where they need a scan; it keeps its per-tile partial sums in a
file-scope device array.  This file is named to be collected last.
"""
import ctypes
import os

import numpy as np
import pytest

from slosh_b200 import _lib
from slosh_b200._lib import SloshConfig, SLOSH_E_CAPACITY

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _ctx(lib, capacity):
    cfg = SloshConfig(3, 0.1, capacity, 1, 0, 0)
    ctx = ctypes.c_void_p()
    assert lib.slosh_ctx_create(ctypes.byref(cfg), ctypes.byref(ctx)) == 0
    return ctx


def _reference_scan(lib, ctx, v):
    out = np.zeros_like(v)
    assert lib.slosh_prefix_sum(ctx, v.ctypes.data, out.ctypes.data, len(v)) == 0
    return out


def _noalloc_scan(lib, torch, v):
    dev_in = torch.from_numpy(v.view(np.int32)).cuda()
    dev_out = torch.empty_like(dev_in)
    assert lib.slosh_prefix_sum_noalloc(dev_in.data_ptr(), dev_out.data_ptr(), len(v), None) == 0
    torch.cuda.synchronize()
    return dev_out.cpu().numpy().view(np.uint32)


def test_noalloc_prefix_sum_matches_context_scan(cuda_lib):
    import torch

    torch.cuda.set_device(0)
    lib = cuda_lib
    ctx = _ctx(lib, 1 << 17)  # context scan accepts up to 2 * 131072 values
    try:
        g = np.load(os.path.join(GOLDEN, "prefix_sum.npz"))
        n = 15071
        rng = np.random.default_rng(21)
        inputs = [
            np.ones(n, np.uint32),
            np.arange(n, dtype=np.uint32),
            g["input"],
            rng.integers(0, 10_000, size=250_000, dtype=np.uint32),  # 62 tiles
            rng.integers(0, 3, size=4097, dtype=np.uint32),  # one element past a tile
        ]
        # two calls in a row per input: the shared scratch keeps the previous
        # call's partial sums and must not leak into the next result
        for v in inputs:
            ref = _reference_scan(lib, ctx, v)
            first = _noalloc_scan(lib, torch, v)
            second = _noalloc_scan(lib, torch, v)
            assert np.array_equal(first, ref)
            assert np.array_equal(second, ref)
        assert np.array_equal(_noalloc_scan(lib, torch, g["input"]), g["expected"])
    finally:
        lib.slosh_ctx_destroy(ctx)


def _numpy_scan(v):
    """Exclusive scan in u32 arithmetic (wraps at 2^32 like the device sums)."""
    out = np.zeros_like(v)
    np.cumsum(v[:-1], dtype=np.uint32, out=out[1:])
    return out


def test_noalloc_prefix_sum_large_and_wrapping(cuda_lib):
    """Inputs beyond the context scan's size: more than 256 tiles (several
    rounds of the tile-sum carry), the maximum size, and totals that wrap
    past 2^32, each scanned twice in a row."""
    import torch

    torch.cuda.set_device(0)
    rng = np.random.default_rng(22)
    cases = [
        rng.integers(0, 1000, size=1_050_000, dtype=np.uint32),  # 257 tiles
        rng.integers(0, 1000, size=5_000_003, dtype=np.uint32),  # 1221 tiles, ragged end
        rng.integers(0, 4, size=67_108_864, dtype=np.uint32),  # the maximum n
        rng.integers(1 << 30, 1 << 31, size=300_001, dtype=np.uint32),  # total wraps 2^32 many times
    ]
    for v in cases:
        ref = _numpy_scan(v)
        assert np.array_equal(_noalloc_scan(cuda_lib, torch, v), ref), len(v)
        assert np.array_equal(_noalloc_scan(cuda_lib, torch, v), ref), len(v)
        torch.cuda.empty_cache()


def test_noalloc_prefix_sum_rejects_oversize(cuda_lib):
    import torch

    torch.cuda.set_device(0)
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros_like(buf)
    # the size check happens before any launch, so the short buffers are never read
    code = cuda_lib.slosh_prefix_sum_noalloc(buf.data_ptr(), out.data_ptr(), 67_108_865, None)
    assert code == SLOSH_E_CAPACITY
    assert cuda_lib.slosh_prefix_sum_noalloc(buf.data_ptr(), out.data_ptr(), 16, None) == 0
    torch.cuda.synchronize()
    assert int(out.sum().item()) == 0

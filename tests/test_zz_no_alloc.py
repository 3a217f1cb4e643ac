"""The allocation-free radix sort entry point (olc_radix_sort_pairs_noalloc).

Callers that cannot allocate device memory when they need a sort (code
running under CUDA graph capture, serving loops held to a fixed memory
budget, hosts whose allocator belongs to another runtime) use this variant;
its scratch is a fixed file-scope device array inside the library.  The test
compares it through the C ABI with the allocating olc_radix_sort_pairs on two
calls in a row (the second smaller than the first, so leftovers of the first
call in the shared array must not leak into the second), and checks that a
request beyond the 1,048,576-pair limit is refused.  Integer sort: results
must match exactly.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _sort_with_context(lib, keys, values, bits):
    import torch

    from ordinarylight_b200 import _native

    cfg = _native.OlcConfig()
    cfg.mode = _native.MODE_REFERENCE_COMPATIBLE
    cfg.max_bounces = 1
    ctx = ctypes.c_void_p()
    _native.check(lib, None, lib.olc_create(ctypes.byref(cfg), ctypes.byref(ctx)))
    try:
        k = torch.as_tensor(keys.view(np.int32).copy(), device="cuda")
        v = torch.as_tensor(values.view(np.int32).copy(), device="cuda")
        torch.cuda.synchronize()
        _native.check(lib, ctx, lib.olc_radix_sort_pairs(ctx, len(keys), bits, _native.ptr(k), _native.ptr(v)))
        return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)
    finally:
        lib.olc_destroy(ctx)


def _sort_without_allocation(lib, keys, values, bits):
    import torch

    from ordinarylight_b200 import _native

    k = torch.as_tensor(keys.view(np.int32).copy(), device="cuda")
    v = torch.as_tensor(values.view(np.int32).copy(), device="cuda")
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    status = lib.olc_radix_sort_pairs_noalloc(len(keys), bits, _native.ptr(k), _native.ptr(v),
                                              ctypes.c_void_p(stream.cuda_stream))
    _native.check(lib, None, status)
    stream.synchronize()
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_the_allocating_sort_on_two_calls(native_library, cuda_device):
    rng = np.random.default_rng(2024)
    for n, bits in ((MAX_PAIRS, 30), (300_001, 32)):
        pool = rng.integers(0, 1 << bits, size=max(2, n // 16), dtype=np.uint64)
        keys = rng.choice(pool, size=n).astype(np.uint32)
        values = np.arange(n, dtype=np.uint32)
        expected = _sort_with_context(native_library, keys, values, bits)
        got = _sort_without_allocation(native_library, keys, values, bits)
        np.testing.assert_array_equal(got[0], expected[0])
        np.testing.assert_array_equal(got[1], expected[1])
        np.testing.assert_array_equal(got[1], np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.parametrize("n,bits", [(1, 8), (2, 24), (2047, 8), (2047, 24), (2048, 24), (5000, 16)])
def test_noalloc_sort_on_a_side_stream_with_odd_pass_counts(native_library, cuda_device, n, bits):
    """Key widths of 8 and 24 bits take one and three digit passes, so the
    sorted pairs end in the scratch array and are copied back; sizes at and
    below one 2,048-key tile; the call is ordered on a side stream that is
    not the default one.  Against a stable host sort."""
    import torch

    from ordinarylight_b200 import _native

    rng = np.random.default_rng(n * 31 + bits)
    pool = rng.integers(0, 1 << bits, size=max(2, n // 4), dtype=np.uint64)     # repeated keys test stability
    keys = rng.choice(pool, size=n).astype(np.uint32)
    values = rng.permutation(n).astype(np.uint32)
    side = torch.cuda.Stream()
    k = torch.as_tensor(keys.view(np.int32).copy(), device="cuda")
    v = torch.as_tensor(values.view(np.int32).copy(), device="cuda")
    torch.cuda.synchronize()
    status = native_library.olc_radix_sort_pairs_noalloc(n, bits, _native.ptr(k), _native.ptr(v),
                                                         ctypes.c_void_p(side.cuda_stream))
    _native.check(native_library, None, status)
    side.synchronize()
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(k.cpu().numpy().view(np.uint32), keys[order])
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint32), values[order])


def test_noalloc_sort_rejects_requests_beyond_its_limit(native_library, cuda_device):
    from ordinarylight_b200 import _native

    status = native_library.olc_radix_sort_pairs_noalloc(MAX_PAIRS + 1, 30, None, None, None)
    assert status == _native.OLC_ERR_VALUE
    assert b"1048576" in native_library.olc_last_error(None)

"""The allocation-free sort entry point (strata_sort_u32_noalloc).

It exists for callers that cannot allocate device memory (host callbacks,
embedders whose allocator owns the device, loops that must not enter the
allocator): it sorts caller-owned buffers with a fixed scratch array inside
the library.  This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes on its own in a
fresh process.  Results must equal the allocating sort (strata_op_sort)
exactly: integer keys leave no tolerance.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 20  # STRATA_NOALLOC_SORT_MAX_KEYS


def _sort_noalloc(lib, torch, keys_np, bits):
    n = len(keys_np)
    src = torch.from_numpy(keys_np.view(np.int32)).cuda()
    dst = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.strata_sort_u32_noalloc(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), n, bits,
                                     C.c_void_p(stream))
    out = dst.cpu().numpy().view(np.uint32)[:n].copy()
    # the input buffer is left unchanged
    assert np.array_equal(src.cpu().numpy().view(np.uint32), keys_np)
    return rc, out


def _sort_allocating(engine, torch, keys_np, bits):
    n = len(keys_np)
    src = torch.from_numpy(keys_np.view(np.int32)).cuda()
    dst = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    engine._check(engine.lib.strata_op_sort(engine.ctx, 4, 0, C.c_void_p(src.data_ptr()), None,
                                            C.c_void_p(dst.data_ptr()), None, n, bits))
    return dst.cpu().numpy().view(np.uint32)[:n].copy()


def test_noalloc_sort_matches_allocating_sort_twice_in_a_row():
    import torch

    import strata_b200 as S
    from strata_b200 import _lib as L
    lib = L.load()
    eng = S.Engine(0)
    try:
        rng = np.random.default_rng(2024)
        # Two calls in a row with different sizes and key widths: the second
        # must not see anything the first left in the shared scratch array.
        for n, bits in ((MAX_KEYS, 26), (300_001, 17)):
            keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
            rc, got = _sort_noalloc(lib, torch, keys, bits)
            assert rc == L.OK
            want = _sort_allocating(eng, torch, keys, bits)
            assert np.array_equal(got, want)
            assert np.array_equal(got, np.sort(keys, kind="stable"))
    finally:
        eng.close()


def test_noalloc_sort_small_and_edge_cases():
    import torch

    import strata_b200 as S
    from strata_b200 import _lib as L
    lib = L.load()
    eng = S.Engine(0)
    try:
        rng = np.random.default_rng(7)
        # one key; key_bits 0 (a plain copy: the output equals the input);
        # the full 32-bit range
        for n, bits in ((1, 12), (1000, 0), (65_537, 32), (4097, 8)):
            hi = 1 << max(bits, 1)
            keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
            rc, got = _sort_noalloc(lib, torch, keys, bits)
            assert rc == L.OK
            want = keys.copy() if bits == 0 else np.sort(keys, kind="stable")
            assert np.array_equal(got, want)
            if bits:
                assert np.array_equal(got, _sort_allocating(eng, torch, keys, bits))
        # the legacy default stream (NULL), as the header allows
        keys = rng.integers(0, 1 << 20, 50_000, dtype=np.uint64).astype(np.uint32)
        src = torch.from_numpy(keys.view(np.int32)).cuda()
        dst = torch.empty(len(keys), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert lib.strata_sort_u32_noalloc(C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()),
                                           len(keys), 20, None) == L.OK
        assert np.array_equal(dst.cpu().numpy().view(np.uint32), np.sort(keys))
    finally:
        eng.close()


def test_noalloc_sort_rejects_oversized_or_overlapping_input():
    import torch

    from strata_b200 import _lib as L
    lib = L.load()
    buf = torch.zeros(64, dtype=torch.int32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    assert lib.strata_sort_u32_noalloc(p, C.c_void_p(buf.data_ptr() + 128), MAX_KEYS + 1, 20, None) == L.E_INVALID
    assert lib.strata_sort_u32_noalloc(p, C.c_void_p(buf.data_ptr() + 128), 8, 33, None) == L.E_INVALID
    # in place, and partly overlapping ranges, are refused (17 bits = an odd
    # pass count, the case that would scatter into the buffer being read)
    assert lib.strata_sort_u32_noalloc(p, p, 16, 17, None) == L.E_INVALID
    assert lib.strata_sort_u32_noalloc(p, C.c_void_p(buf.data_ptr() + 32), 16, 17, None) == L.E_INVALID
    assert lib.strata_sort_u32_noalloc(C.c_void_p(buf.data_ptr() + 32), p, 16, 17, None) == L.E_INVALID
    # adjacent, non-overlapping ranges are fine
    assert lib.strata_sort_u32_noalloc(p, C.c_void_p(buf.data_ptr() + 64), 16, 17, None) == L.OK

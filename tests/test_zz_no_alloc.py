"""EZmockB200_mt19937_fill_noalloc: the MT19937 fill with static device scratch.

It must give the same draws as the allocating entry point EZmockB200_rng_raw
(randgen 1) and as the CPU oracle's MT19937 stream, call after call, and
reject requests larger than its scratch before touching the GPU.  This file
is named to be collected last, so the GPU test also runs after every other
test has used the library in the process.
"""
import ctypes

import numpy as np
import pytest

from ezmock_b200 import _lib
from oracle.pyoracle import Oracle

MAX_DRAWS = 1 << 47
ERR_SCRATCH_SIZE = 64
ERR_ARG_NULL = 12


def _rng_raw(L, seed, start, n):
    out = np.empty(n, np.uint32)
    assert L.EZmockB200_rng_raw(1, seed, start, n, out.ctypes.data_as(ctypes.c_void_p)) == 0
    return out


def test_noalloc_rejects_oversize_requests():
    L = _lib.load(32)
    dummy = ctypes.c_void_p(16)           # never dereferenced: rejected first
    assert L.EZmockB200_mt19937_fill_noalloc(1, 0, MAX_DRAWS + 1, dummy, None) == ERR_SCRATCH_SIZE
    assert L.EZmockB200_mt19937_fill_noalloc(1, (1 << 64) - 10, 100, dummy, None) == ERR_SCRATCH_SIZE
    assert L.EZmockB200_mt19937_fill_noalloc(1, 0, 10, None, None) == ERR_ARG_NULL
    assert L.EZmockB200_mt19937_fill_noalloc(1, 0, 0, None, None) == 0
    msg = L.EZmock_errmsg(ERR_SCRATCH_SIZE).decode()
    assert "static scratch" in msg


@pytest.mark.gpu
def test_noalloc_matches_allocating_fill():
    import torch
    L = _lib.load(32)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    cases = [
        (12345, 1000, 70_001),             # one chunk
        (7, 3 * 2**20 + 5, 5_000_000),     # several chunks, doubling levels
        (2**40 + 3, 2**33 + 17, 300_000),  # 64-bit seed (init_by_array seeding)
    ]
    bufs = [torch.empty(n, dtype=torch.int32, device="cuda") for _, _, n in cases]
    # back-to-back calls on one stream: each reuses the same static scratch
    for (seed, start, n), b in zip(cases, bufs):
        e = L.EZmockB200_mt19937_fill_noalloc(seed, start, n, ctypes.c_void_p(b.data_ptr()),
                                              ctypes.c_void_p(stream.cuda_stream))
        assert e == 0, L.EZmock_errmsg(e).decode()
    torch.cuda.synchronize()
    O = Oracle(64)
    for (seed, start, n), b in zip(cases, bufs):
        got = b.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got, _rng_raw(L, seed, start, n))
        # independently of the library's jump tables and generation kernels
        np.testing.assert_array_equal(got, O.rng_raw(1, seed, start, n))
    # again, on the legacy default stream, into the first buffer
    seed, start, n = cases[1]
    b = bufs[1]
    b.zero_()
    torch.cuda.synchronize()
    assert L.EZmockB200_mt19937_fill_noalloc(seed, start, n, ctypes.c_void_p(b.data_ptr()),
                                             None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(b.cpu().numpy().view(np.uint32), _rng_raw(L, seed, start, n))

"""The allocation-free Morton entry point against the allocating one.

tlr_morton_order_noalloc exists for callers that may not allocate device memory during the
call (for example while another framework's caching allocator owns the device's memory, or in
a service loop that allocates nothing after start-up).  It keeps its working memory in one
fixed array inside the library, shared by every call, so these checks run two calls in a row:
the second must not be disturbed by what the first left in that array.  Morton ordering is
integer work, so the permutations must be identical.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from adaptive_tlr_pilots_b200 import _lib as L
    return L, L.load()


def _points(n, seed):
    xy = np.random.default_rng(seed).random((n, 2))
    xy[::5] = xy[1::5][: len(xy[::5])]          # repeated sites: ties keep input order
    xy[3] = [0.0, 1.0]
    xy[4] = [1.5, -0.25]                         # outside the unit square: clipped
    return xy


def test_noalloc_matches_allocating_entry_point_twice_in_a_row():
    import torch
    L, lib = _lib()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    cases = [_points(60000, 11), _points(2345, 12)]
    xs = [torch.from_numpy(c).to(dev) for c in cases]
    want = []
    for x in xs:
        p = torch.empty(x.shape[0], dtype=torch.int64, device=dev)
        L.check(lib.tlr_morton_order(ctypes.c_void_p(x.data_ptr()), x.shape[0], 10, ctypes.c_void_p(p.data_ptr()),
                                     stream))
        want.append(p.cpu().numpy())
    got = []
    for x in xs:  # two calls in a row on the shared array
        p = torch.empty(x.shape[0], dtype=torch.int64, device=dev)
        L.check(lib.tlr_morton_order_noalloc(ctypes.c_void_p(x.data_ptr()), x.shape[0], 10,
                                             ctypes.c_void_p(p.data_ptr()), stream))
        got.append(p)
    torch.cuda.synchronize()
    for w, g in zip(want, got):
        np.testing.assert_array_equal(g.cpu().numpy(), w)


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch
    L, lib = _lib()
    x = torch.zeros((4, 2), dtype=torch.float64, device="cuda")
    p = torch.empty(4, dtype=torch.int64, device="cuda")
    rc = lib.tlr_morton_order_noalloc(ctypes.c_void_p(x.data_ptr()), (1 << 20) + 1, 10,
                                      ctypes.c_void_p(p.data_ptr()), None)
    assert rc == -1 and "1048576" in L.last_error()
    rc = lib.tlr_morton_order_noalloc(ctypes.c_void_p(x.data_ptr()), 4, 11, ctypes.c_void_p(p.data_ptr()), None)
    assert rc == -1

"""Failure detection without a GPU fault: the tensor-core kernels' waits are bounded, and a wait
that runs out ends its kernel with TLR_ERR_TIMEOUT, its tensor memory freed, the context usable.
The wait is made to run out on an mbarrier phase that nothing completes (no trap, no bad address)."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def tlr():
    import adaptive_tlr_pilots_b200 as m
    yield m
    m.release_plans()


def test_bounded_wait_runs_out_and_context_stays_usable(tlr):
    from adaptive_tlr_pilots_b200 import _lib
    lib = _lib.load()
    polls = 4096
    ms, limit = ctypes.c_double(0.0), ctypes.c_longlong(0)
    rc = lib.tlr_selftest_bounded_wait(polls, 0, ctypes.byref(ms), ctypes.byref(limit))
    assert rc == -7, (rc, _lib.last_error())                 # TLR_ERR_TIMEOUT, reported to the host
    assert "ran out" in _lib.last_error()
    per_poll_s = ms.value / 1e3 / polls
    print(f"bounded wait: {per_poll_s * 1e9:.0f} ns per poll, production limit {limit.value} polls "
          f"= {limit.value * per_poll_s:.2f} s")
    assert limit.value * per_poll_s <= 3.0                    # a stuck wait ends within a second or two
    # the context is intact: a normal evaluation right after gives the golden result
    d = np.load(os.path.join(GOLD, "n1030_b100_data.npz"))
    ll, _, info = tlr.tlr_loglik(d["S"], d["y"], (1.0, 0.3, 0.05), tlr.tile_bounds(1030, 100), "adaptive", 0.9)
    assert ll is not None and info["completed"]
    ll2, g, _ = tlr.tlr_loglik_grad(d["S"], d["y"], (1.0, 0.3, 0.05), tlr.tile_bounds(1030, 100), "adaptive", 0.9,
                                    precision="mixed")          # the tensor-core kernel itself runs again
    assert g is not None and abs(ll2 - ll) < 1e-6 * abs(ll)

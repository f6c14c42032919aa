"""Failure detection without a GPU fault.  Every device wait of the tile
kernel (bulk-copy and tensor-core completions) is bounded; the self-test
runs that same wait on a barrier that nothing completes, with a short
limit, and checks that it gives up, reports, and leaves the context usable.
Host-side failures (malformed programs, oversized requests, cancellation)
are covered beside the features they belong to."""
import ctypes
import time

import numpy as np
import pytest

from oracle import oracle
from qlassical_b200 import _lib, circuits


def test_selftest_rejects_bad_limits():
    flag = ctypes.c_int(0)
    for bad in (0, 5000):
        with pytest.raises(ValueError):
            _lib.call("qlb_selftest_bounded_wait", bad, ctypes.byref(flag))


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_context_survives():
    import qlassical_b200 as q
    flag = ctypes.c_int(0)
    t0 = time.perf_counter()
    _lib.call("qlb_selftest_bounded_wait", 50, ctypes.byref(flag))
    dt = time.perf_counter() - t0
    assert flag.value == 1
    assert 0.04 < dt < 1.5
    m = circuits.random_h_rx_cx(14, 6, seed=3)
    eng = q.CUDAEngine(14, mode="tiled")
    eng.execute(m)
    want, _ = oracle.run_oracle(m)
    assert oracle.infidelity(want, eng.state()) < 1e-6

"""qlb_expect_z_noalloc: the allocation-free <Z_q> reduction for callers
that must not allocate device memory (e.g. a serving loop that accounts all
free HBM to resident requests).  It must give the same values as the
allocating entry point (qlb_engine_expect_z), on consecutive calls that
reuse its fixed scratch array, and reject sizes beyond its scratch limit.
This file sorts last so a run that stops at the first failure has already
run every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import _lib, circuits

pytestmark = pytest.mark.gpu

TOL = 1e-12   # both paths reduce in FP64 over the same complex64 state


def _noalloc(engine, n):
    L = _lib.lib()
    fn = L.qlb_expect_z_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    out = np.full(n, np.nan)
    _lib.check(fn(engine.device_state(), n, out.ctypes.data, engine.stream()))
    return out


def _free_bytes():
    free = ctypes.c_uint64()
    total = ctypes.c_uint64()
    sm = ctypes.c_int()
    _lib.call("qlb_device_info", ctypes.byref(sm), ctypes.byref(free), ctypes.byref(total))
    return free.value


def test_noalloc_takes_no_memory_after_its_warm_up_call():
    """The first call commits the fixed scratch; later calls change the
    device's free memory by nothing."""
    n = 18
    e = q.CUDAEngine(n, seed=1)
    e.execute(circuits.random_rot_cz(n, 3, seed=2))
    e.expect_z()             # the allocating path's scratch exists before we measure
    _noalloc(e, n)           # warm-up: commits the scratch on this device
    e.synchronize()
    before = _free_bytes()
    for _ in range(3):
        _noalloc(e, n)
    assert _free_bytes() == before


@pytest.mark.parametrize("n", [9, 22, 16])
def test_noalloc_matches_allocating_reduction_twice(n):
    m = circuits.random_rot_cz(n, 4, seed=n)
    e = q.CUDAEngine(n, seed=1)
    e.execute(m)
    want = e.expect_z()
    first = _noalloc(e, n)
    second = _noalloc(e, n)
    assert np.max(np.abs(first - want)) <= TOL
    assert np.max(np.abs(second - want)) <= TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    e = q.CUDAEngine(4, seed=1)
    L = _lib.lib()
    fn = L.qlb_expect_z_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    out = np.zeros(40)
    with pytest.raises(ValueError):
        _lib.check(fn(e.device_state(), 35, out.ctypes.data, e.stream()))
    with pytest.raises(ValueError):
        _lib.check(fn(e.device_state(), 0, out.ctypes.data, e.stream()))

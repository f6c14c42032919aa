"""Batched mode: many independent circuits per launch (qlb_batch_* in the C ABI).

Each circuit runs from |0...0> and reports <Z_q> for its qubits (FP64
reduction), exactly as CUDAEngine.execute() followed by expect_z() would,
but all circuits advance together: one tile-kernel launch per pass round
over a work list of (state, pass) entries, captured with the |0...0>
set-up and the reductions into one CUDA graph.  ``mode="auto"`` autotunes:
six planner configurations -- FP32 CUDA-core or tensor-core fused tiles,
times 3, 4 or 5 fixed low tile qubits -- are timed on a sample of each size
class (circuits of one padded qubit count); the mode is chosen for the whole
batch (a round runs one kernel body) and the fixed low qubits per class;
``stats()["tune"]`` reports the search.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import call, lib
from .ir import IRModule

_MODES = {"tiled": _lib.MODE_TILED, "tiled_tc": _lib.MODE_TILED_TC, "auto": -1}
_MODE_NAMES = {_lib.MODE_TILED: "tiled", _lib.MODE_TILED_TC: "tiled_tc", -1: "per size class"}


class Batch:
    """A planned batch; run() launches it, expect_z() reads the results."""

    def __init__(self, modules: Sequence[IRModule], mode: str = "auto", fuse: int = 0):
        """fuse: blocks of up to this many qubits (<= 5) formed by the GPU
        middle end in each circuit before planning (0: no fusion); fused
        blocks run on the tensor cores."""
        if not modules:
            raise ValueError("empty batch")
        self._h = None
        m = _MODES[mode] if isinstance(mode, str) else int(mode)
        progs, keep, pools = [], [], []
        for mod in modules:
            p = np.ascontiguousarray(mod.program(), dtype=_lib.GATE_INSTR_DTYPE)
            pv, k = mod.unitaries().view()
            progs.append(p)
            keep.append(k)
            pools.append(pv)
        n = len(modules)
        prog_ptrs = (ctypes.c_void_p * n)(*[p.ctypes.data if p.size else None for p in progs])
        counts = (ctypes.c_uint64 * n)(*[p.size for p in progs])
        pool_arr = (_lib.PoolView * n)(*pools)
        nq = (ctypes.c_uint32 * n)(*[int(mod.num_qubits) for mod in modules])
        h = ctypes.c_void_p()
        call("qlb_batch_create_ex", ctypes.byref(h), n, ctypes.cast(prog_ptrs, ctypes.c_void_p),
             ctypes.cast(counts, ctypes.c_void_p), ctypes.cast(pool_arr, ctypes.c_void_p),
             ctypes.cast(nq, ctypes.c_void_p), m, int(fuse))
        self._h = h
        self._n = n
        self._nq = [int(mod.num_qubits) for mod in modules]
        del keep

    def __del__(self):
        if getattr(self, "_h", None):
            lib().qlb_batch_destroy(self._h)
            self._h = None

    def __len__(self) -> int:
        return self._n

    def run(self) -> None:
        """One graph launch (asynchronous)."""
        call("qlb_batch_run", self._h)

    def synchronize(self) -> None:
        call("qlb_batch_synchronize", self._h)

    def expect_z(self) -> list[np.ndarray]:
        """<Z_q> per circuit (after synchronize())."""
        stride = max(self._nq)
        out = np.zeros((self._n, stride), dtype=np.float64)
        call("qlb_batch_expect_z", self._h, out.ctypes.data, stride)
        return [out[c, :self._nq[c]].copy() for c in range(self._n)]

    def state(self, index: int) -> np.ndarray:
        dim = 1 << self._nq[index]
        out = np.empty(dim, dtype=np.complex128)
        call("qlb_batch_state", self._h, int(index), out.ctypes.data, dim)
        return out

    def stats(self) -> dict:
        info = _lib.BatchInfo()
        call("qlb_batch_stats", self._h, ctypes.byref(info))
        return {
            "circuits": info.circuits, "rounds": info.rounds, "mode": _MODE_NAMES.get(info.mode, info.mode),
            "launches": info.launches, "tiles": info.tiles, "passes": info.passes,
            "amp_updates": info.amp_updates, "state_bytes": info.state_bytes,
            "autotune_ms": list(info.autotune_ms),
            "tune_seconds": info.tune_seconds,
            "fuse_seconds": info.fuse_seconds,
            "plan_seconds": info.plan_seconds,
            "tune": [{"num_qubits": t.num_qubits, "circuits": t.circuits, "sample": t.sample,
                      "best": _lib.batch_tune_candidate(t.best),
                      "ms": [float(x) for x in t.ms]}
                     for t in info.tune[:info.tune_classes]],
        }

    def stream(self) -> int:
        s = ctypes.c_void_p()
        call("qlb_batch_stream", self._h, ctypes.byref(s))
        return s.value or 0


def run_batch(modules: Sequence[IRModule], mode: str = "auto", fuse: int = 0) -> list[np.ndarray]:
    """Plans, runs and returns <Z_q> of every circuit."""
    b = Batch(modules, mode, fuse)
    b.run()
    b.synchronize()
    return b.expect_z()

"""Serving loop (qlb_server_* in the C ABI): continuous batching of circuit
requests on one GPU.

A request is (circuit, shots, seed), run from |0...0>; its result is <Z_q>
for every qubit (FP64) and `shots` sampled basis states.  submit() plans the
circuit on the calling thread and queues it; the server thread admits
queued requests in arrival order while their state vectors fit a device
arena reserved at start-up, advances every admitted request by one tile pass
per round (one launch per round over all of them) and finishes each with its
reduction and sampling.  A request's results do not depend on the other
requests in flight.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import call, lib
from .ir import IRModule


@dataclass
class Result:
    expect_z: np.ndarray
    samples: np.ndarray
    num_qubits: int
    passes: int
    t_submit: float
    t_admit: float
    t_done: float

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    def __init__(self, memory_bytes: int = 0, mode: str = "tiled", max_active: int = 0, fuse_from: int = 0):
        """fuse_from: requests of at least this many qubits are fused by the
        GPU middle end (blocks of up to 5 qubits) and planned for the tensor
        cores; the others run in `mode`.  0: no fusion."""
        cfg = _lib.ServerConfig(int(memory_bytes), _lib.MODE_TILED_TC if mode == "tiled_tc" else _lib.MODE_TILED,
                                int(max_active), int(fuse_from), 0)
        h = ctypes.c_void_p()
        call("qlb_server_create", ctypes.byref(h), ctypes.byref(cfg))
        self._h = h
        self._meta = {}

    def submit(self, module: IRModule, shots: int = 1024, seed: int = 0) -> int:
        prog = np.ascontiguousarray(module.program(), dtype=_lib.GATE_INSTR_DTYPE)
        pv, keep = module.unitaries().view()
        rid = ctypes.c_uint64()
        call("qlb_server_submit", self._h, prog.ctypes.data if prog.size else None, prog.size, ctypes.byref(pv),
             int(module.num_qubits), int(shots), int(seed), ctypes.byref(rid))
        del keep
        self._meta[rid.value] = (int(module.num_qubits), int(shots))
        return rid.value

    def wait(self, rid: int, timeout: float = 600.0) -> None:
        call("qlb_server_wait", self._h, int(rid), float(timeout))

    def cancel(self, rid: int) -> None:
        """A queued request leaves at once, an admitted one at the next round
        boundary; wait() / result() then raise RuntimeError."""
        call("qlb_server_cancel", self._h, int(rid))

    def result(self, rid: int, timeout: float = 600.0) -> Result:
        self.wait(rid, timeout)
        n, shots = self._meta.pop(rid)
        ez = np.zeros(n, dtype=np.float64)
        smp = np.zeros(shots, dtype=np.uint64)
        info = _lib.RequestInfo()
        call("qlb_server_result", self._h, int(rid), ez.ctypes.data, n, smp.ctypes.data if shots else None, shots,
             ctypes.byref(info))
        return Result(ez, smp, info.num_qubits, info.passes, info.t_submit, info.t_admit, info.t_done)

    def stats(self) -> dict:
        s = _lib.ServerInfo()
        call("qlb_server_stats", self._h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in _lib.ServerInfo._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            call("qlb_server_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

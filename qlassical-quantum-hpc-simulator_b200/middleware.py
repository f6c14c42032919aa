"""Middle end for the GPU backend: Python mirror of Qlassical's Middleware /
TranspilerConfig / cost models (include/middleware/middleware.hpp:33-132,
352-481) over the native transpile_gpu (csrc/middle_end.cpp)."""
from __future__ import annotations

import ctypes
import dataclasses
import enum
from typing import Callable, Optional

import numpy as np

from . import _lib
from ._lib import call, lib
from .ir import IRModule, UnitaryPool


class Backend(enum.IntEnum):
    CPU_OPENMP = 0x00
    MPI = 0x01
    GPU = 0x02


class CostModelType(enum.IntEnum):
    THRESHOLD = 0
    GREEDY = 1
    CUSTOM = 2


class WindowingCostModel:
    """evaluate_swap(freq, log_to_phys, phys_to_log) -> (active, victim) | None."""

    def evaluate_swap(self, window_frequencies, log_to_phys, phys_to_log):
        raise NotImplementedError

    def get_k_safe(self) -> int:
        raise NotImplementedError


@dataclasses.dataclass
class TranspilerConfig:
    """TranspilerConfig (middleware.hpp:362-386) plus the GPU fusion width."""
    enable_gate_fusion: bool = True
    enable_hw_awareness: bool = True
    cost_model_type: CostModelType = CostModelType.THRESHOLD
    numa_penalty: int = 10
    swap_penalty: int = 1
    k_safe: Optional[int] = None
    custom_cost_model: Optional[WindowingCostModel] = None
    max_fusion_qubits: int = 5
    reference_fusable_set: bool = False

    def set_cost_model(self, model: WindowingCostModel) -> None:
        self.custom_cost_model = model
        self.cost_model_type = CostModelType.CUSTOM


_COST_FN = _lib.COST_MODEL_FN
_TranspileConfigC = _lib.TranspileConfig


def gpu_safe_qubit_limit() -> int:
    """GPUTopology::get_safe_qubit_limit(): qubits held by one on-chip tile."""
    v = ctypes.c_uint32()
    call("qlb_gpu_safe_qubit_limit", ctypes.byref(v))
    return v.value


class Middleware:
    """Middleware::transpile (middleware.hpp:466-481) for Backend.GPU."""

    def transpile(self, module: IRModule, backend: Backend = Backend.GPU,
                  config: Optional[TranspilerConfig] = None) -> IRModule:
        if backend != Backend.GPU:
            raise ValueError("this package provides the GPU middle end only (Backend.GPU)")
        config = config or TranspilerConfig()
        L = lib()
        c = _TranspileConfigC()
        c.enable_gate_fusion = int(config.enable_gate_fusion)
        c.enable_hw_awareness = int(config.enable_hw_awareness)
        c.cost_model_type = int(config.cost_model_type)
        c.numa_penalty = int(config.numa_penalty)
        c.swap_penalty = int(config.swap_penalty)
        model = config.custom_cost_model
        k_safe = config.k_safe
        if k_safe is None and model is not None:
            k_safe = model.get_k_safe()
        c.k_safe = -1 if k_safe is None else int(k_safe)
        c.max_fusion_qubits = int(config.max_fusion_qubits)
        c.reference_fusable_set = int(config.reference_fusable_set)
        cb = None
        if config.cost_model_type == CostModelType.CUSTOM and model is None:
            raise ValueError("TranspilerConfig: CostModelType::CUSTOM specified but custom_cost_model is null.")
        if model is not None:
            def _cb(ctx, freq, l2p, p2l, n, active, victim):
                f = np.ctypeslib.as_array(freq, shape=(n,)).copy()
                a = np.ctypeslib.as_array(l2p, shape=(n,)).copy()
                b = np.ctypeslib.as_array(p2l, shape=(n,)).copy()
                r = model.evaluate_swap(f, a, b)
                if r is None:
                    return 0
                active[0], victim[0] = int(r[0]), int(r[1])
                return 1
            cb = _COST_FN(_cb)
            c.custom_cost_model = cb
        prog = np.ascontiguousarray(module.program(), dtype=_lib.GATE_INSTR_DTYPE)
        pv, keep = module.unitaries().view()
        h = ctypes.c_void_p()
        fn = L.qlb_transpile_gpu
        fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_lib.PoolView), ctypes.c_uint32,
                       ctypes.POINTER(_TranspileConfigC), ctypes.POINTER(ctypes.c_void_p)]
        _lib.check(fn(_lib.ptr(prog), prog.size, ctypes.byref(pv), module.num_qubits, ctypes.byref(c),
                      ctypes.byref(h)))
        del keep, cb
        try:
            p = ctypes.c_void_p()
            cnt = ctypes.c_uint64()
            call("qlb_module_program", h, ctypes.byref(p), ctypes.byref(cnt))
            out_prog = np.frombuffer(ctypes.string_at(p.value, 16 * cnt.value), dtype=_lib.GATE_INSTR_DTYPE).copy() \
                if cnt.value else np.zeros(0, dtype=_lib.GATE_INSTR_DTYPE)
            pool = _lib.PoolView()
            call("qlb_module_pool", h, ctypes.byref(pool))
            data = (np.frombuffer(ctypes.string_at(pool.data, 16 * pool.num_elements), dtype=np.complex128).copy()
                    if pool.num_elements else np.zeros(0, dtype=np.complex128))
            meta = (np.frombuffer(ctypes.string_at(pool.metadata, 12 * pool.num_matrices),
                                  dtype=_lib.MATRIX_ENTRY_DTYPE).copy()
                    if pool.num_matrices else np.zeros(0, dtype=_lib.MATRIX_ENTRY_DTYPE))
        finally:
            L.qlb_module_destroy(h)
        out = IRModule(module.num_qubits, unitary_pool=UnitaryPool.from_arrays(data, meta))
        out.set_program(out_prog)
        return out

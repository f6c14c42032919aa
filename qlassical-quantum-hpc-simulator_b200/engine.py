"""CUDAStateVector / CUDAEngine: Python mirror of the reference's
StateVector (include/backend/state_vector.hpp:17-47) and ExecutionEngine
(include/backend/execution_engine.hpp:20-79) over the C ABI.  Method names,
argument meaning and error behaviour follow CPUStateVector
(cpu_state_vector.hpp:24-162) and CPUOpenMPEngine (cpu_openmp_engine.hpp:51-672).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import call, lib
from .ir import IRModule, UnitaryPool

MODES = {"plain": _lib.MODE_PLAIN, "tiled": _lib.MODE_TILED, "tiled_tc": _lib.MODE_TILED_TC}


def _as_c128(amps) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(amps, dtype=np.complex128).reshape(-1))
    return a


class CUDAStateVector:
    """complex64 state vector resident in HBM (move-only in C++)."""

    def __init__(self):
        h = ctypes.c_void_p()
        call("qlb_state_create", ctypes.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().qlb_state_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def initialize(self, arg) -> None:
        """initialize(num_qubits) -> |0...0>; initialize(amplitudes) -> checked copy."""
        if isinstance(arg, (int, np.integer)):
            call("qlb_state_initialize", self._h, int(arg))
        else:
            a = _as_c128(arg)
            call("qlb_state_initialize_from", self._h, _lib.ptr(a), a.size)

    def num_qubits(self) -> int:
        v = ctypes.c_uint32()
        call("qlb_state_num_qubits", self._h, ctypes.byref(v))
        return v.value

    def dimension(self) -> int:
        v = ctypes.c_uint64()
        call("qlb_state_dimension", self._h, ctypes.byref(v))
        return v.value

    def empty(self) -> bool:
        v = ctypes.c_int()
        call("qlb_state_empty", self._h, ctypes.byref(v))
        return bool(v.value)

    def amplitudes(self) -> np.ndarray:
        out = np.empty(self.dimension(), dtype=np.complex128)
        call("qlb_state_download", self._h, _lib.ptr(out), out.size)
        return out

    def device_ptr(self) -> int:
        p = ctypes.c_void_p()
        call("qlb_state_device_ptr", self._h, ctypes.byref(p))
        return p.value or 0


class Plan:
    """A compiled program (qlb_plan): run it with CUDAEngine.run(plan)."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().qlb_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def stats(self) -> dict:
        st = _lib.ExecStats()
        call("qlb_plan_stats", self._h, ctypes.byref(st))
        return st.as_dict()


def set_device(device: int) -> None:
    call("qlb_set_device", int(device))


def describe_plan(program, num_qubits: int, mode: str = "tiled", pool: Optional[UnitaryPool] = None,
                  physical_global_swap: bool = False, tile_low: int = 3, tc_chain: bool = True) -> dict:
    """EXPLAIN: the engine's plan for `program` (host-only, no GPU needed).
    tile_low and tc_chain are the planner options QLB_OPT_TILE_LOW and
    QLB_OPT_TC_CHAIN."""
    import json
    if isinstance(program, IRModule):
        pool = program.unitaries()
        program = program.program()
    prog = np.ascontiguousarray(program, dtype=_lib.GATE_INSTR_DTYPE)
    pool = pool if pool is not None else UnitaryPool()
    pv, keep = pool.view()
    L = lib()
    fn = L.qlb_describe_plan_opts
    fn.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.c_uint64, ctypes.POINTER(_lib.PoolView), ctypes.c_char_p, ctypes.c_uint64,
                   ctypes.POINTER(ctypes.c_uint64)]
    fn.restype = ctypes.c_int
    m = MODES[mode] if isinstance(mode, str) else int(mode)
    opts = (num_qubits, m, int(physical_global_swap), int(tile_low), int(bool(tc_chain)), _lib.ptr(prog), prog.size,
            ctypes.byref(pv))
    need = ctypes.c_uint64()
    _lib.check(fn(*opts, None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(need.value)
    _lib.check(fn(*opts, buf, need.value, ctypes.byref(need)))
    del keep
    return json.loads(buf.value.decode())


class CUDAEngine:
    """ExecutionEngine on one B200.

    CUDAEngine(num_qubits, seed=None, reserve_meas=0)          (:65-80)
    CUDAEngine(initial_state=amplitudes, seed=..., ...)        (:87-102)
    CUDAEngine(state_vector=sv)  -- takes ownership, sv empty  (:105-107)
    """

    def __init__(self, num_qubits: Optional[int] = None, seed: Optional[int] = None, reserve_meas: int = 0,
                 initial_state=None, state_vector: Optional[CUDAStateVector] = None, mode: str = "tiled"):
        h = ctypes.c_void_p()
        has_seed = 0 if seed is None else 1
        s = 0 if seed is None else int(seed) & 0xFFFFFFFFFFFFFFFF
        if state_vector is not None:
            call("qlb_engine_create_from_state", ctypes.byref(h), state_vector.handle)
        elif initial_state is not None:
            a = _as_c128(initial_state)
            call("qlb_engine_create_from_amplitudes", ctypes.byref(h), _lib.ptr(a), a.size, has_seed, s,
                 int(reserve_meas))
        else:
            if num_qubits is None:
                raise ValueError("CUDAEngine needs num_qubits, initial_state or state_vector")
            call("qlb_engine_create", ctypes.byref(h), int(num_qubits), has_seed, s, int(reserve_meas))
        self._h = h
        self.set_mode(mode)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().qlb_engine_destroy(h)
            self._h = None

    # -- ExecutionEngine interface ------------------------------------------
    def reset(self, initial_state=None) -> None:
        if initial_state is None:
            call("qlb_engine_reset", self._h)
        else:
            a = _as_c128(initial_state)
            call("qlb_engine_reset_to", self._h, _lib.ptr(a), a.size)

    def set_seed(self, seed: int) -> None:
        call("qlb_engine_set_seed", self._h, int(seed) & 0xFFFFFFFFFFFFFFFF)

    def reserve_measurements(self, count: int) -> None:
        call("qlb_engine_reserve_measurements", self._h, int(count))

    def measurements(self) -> list:
        p = ctypes.c_void_p()
        n = ctypes.c_uint64()
        call("qlb_engine_measurements", self._h, ctypes.byref(p), ctypes.byref(n))
        if n.value == 0:
            return []
        return list(ctypes.string_at(p.value, n.value))

    def execute(self, program, pool: Optional[UnitaryPool] = None) -> None:
        """execute(IRModule) or execute(program_array, pool)."""
        if isinstance(program, IRModule):
            pool = program.unitaries()
            program = program.program()
        prog = np.ascontiguousarray(program, dtype=_lib.GATE_INSTR_DTYPE)
        pool = pool if pool is not None else UnitaryPool()
        pv, keep = pool.view()
        call("qlb_engine_execute", self._h, _lib.ptr(prog), prog.size, ctypes.byref(pv))
        del keep

    def compile(self, program, pool: Optional[UnitaryPool] = None) -> Plan:
        """Compiles a program for this engine's qubit count and mode."""
        if isinstance(program, IRModule):
            pool = program.unitaries()
            program = program.program()
        prog = np.ascontiguousarray(program, dtype=_lib.GATE_INSTR_DTYPE)
        pool = pool if pool is not None else UnitaryPool()
        pv, keep = pool.view()
        h = ctypes.c_void_p()
        call("qlb_engine_compile", self._h, _lib.ptr(prog), prog.size, ctypes.byref(pv), ctypes.byref(h))
        del keep
        return Plan(h)

    def run(self, plan: Plan) -> None:
        """Enqueues a compiled plan on the engine's stream (asynchronous
        unless the plan measures)."""
        call("qlb_engine_run", self._h, plan.handle)

    def state(self) -> np.ndarray:
        """D2H copy widened to complex128 (the reference returns a span)."""
        out = np.empty(1 << self.num_qubits(), dtype=np.complex128)
        call("qlb_engine_state", self._h, _lib.ptr(out), out.size)
        return out

    def num_qubits(self) -> int:
        v = ctypes.c_uint32()
        call("qlb_engine_num_qubits", self._h, ctypes.byref(v))
        return v.value

    # -- engine-specific (cpu_openmp_engine.hpp:110-112, 240-247) -----------
    def set_state_vector(self, sv: CUDAStateVector) -> None:
        call("qlb_engine_set_state_vector", self._h, sv.handle)

    def extract_state_vector(self) -> CUDAStateVector:
        sv = CUDAStateVector()
        call("qlb_engine_extract_state_vector", self._h, sv.handle)
        return sv

    release_state_vector = extract_state_vector

    # -- B200 extras --------------------------------------------------------
    def set_mode(self, mode) -> None:
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        call("qlb_engine_set_mode", self._h, m)

    def mode(self) -> str:
        v = ctypes.c_int()
        call("qlb_engine_get_mode", self._h, ctypes.byref(v))
        return {b: a for a, b in MODES.items()}[v.value]

    def set_option(self, key: int, value: int) -> None:
        call("qlb_engine_set_option", self._h, int(key), int(value))

    def synchronize(self) -> None:
        call("qlb_engine_synchronize", self._h)

    def stream(self) -> int:
        p = ctypes.c_void_p()
        call("qlb_engine_stream", self._h, ctypes.byref(p))
        return p.value or 0

    def device_state(self) -> int:
        p = ctypes.c_void_p()
        call("qlb_engine_device_state", self._h, ctypes.byref(p))
        return p.value or 0

    def last_stats(self) -> dict:
        st = _lib.ExecStats()
        call("qlb_engine_last_stats", self._h, ctypes.byref(st))
        return st.as_dict()

    def norm_sq(self) -> float:
        v = ctypes.c_double()
        call("qlb_engine_norm_sq", self._h, ctypes.byref(v))
        return v.value

    def prob_one(self, qubit: int) -> float:
        v = ctypes.c_double()
        call("qlb_engine_prob_one", self._h, int(qubit), ctypes.byref(v))
        return v.value

    def expect_z(self) -> np.ndarray:
        n = self.num_qubits()
        out = np.empty(n, dtype=np.float64)
        call("qlb_engine_expect_z", self._h, _lib.ptr(out), n)
        return out

    def amplitudes_at(self, indices) -> np.ndarray:
        """Amplitudes at the given basis indices (device-side gather)."""
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        out = np.empty(idx.size, dtype=np.complex128)
        call("qlb_engine_amplitudes_at", self._h, idx.ctypes.data if idx.size else None, idx.size,
             out.ctypes.data if idx.size else None)
        return out

    def sample(self, seed: int, shots: int) -> np.ndarray:
        out = np.empty(int(shots), dtype=np.uint64)
        call("qlb_engine_sample", self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, int(shots), _lib.ptr(out))
        return out


class Check64:
    """The FP64 checker (qlb_check64_*): a complex128 device state that runs
    a program gate by gate in double precision, and compares itself with a
    complex64 device state over the whole vector (max |delta| and
    infidelity, reduced in FP64)."""

    def __init__(self, num_qubits: int):
        h = ctypes.c_void_p()
        call("qlb_check64_create", ctypes.byref(h), int(num_qubits))
        self._h = h
        self.n = int(num_qubits)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().qlb_check64_destroy(h)
            self._h = None

    def close(self) -> None:
        self.__del__()

    def execute(self, program, pool: Optional[UnitaryPool] = None) -> None:
        if isinstance(program, IRModule):
            pool = program.unitaries()
            program = program.program()
        prog = np.ascontiguousarray(program, dtype=_lib.GATE_INSTR_DTYPE)
        pool = pool if pool is not None else UnitaryPool()
        pv, keep = pool.view()
        call("qlb_check64_execute", self._h, _lib.ptr(prog), prog.size, ctypes.byref(pv))
        del keep

    def compare(self, engine: "CUDAEngine") -> dict:
        """Compares with the engine's current device state (same size)."""
        if engine.num_qubits() != self.n:
            raise ValueError("the engine's qubit count differs from the checker's")
        engine.synchronize()
        r = _lib.Check64Result()
        call("qlb_check64_compare", self._h, ctypes.c_void_p(engine.device_state()), ctypes.byref(r))
        return r.as_dict()

    def state(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.complex128)
        call("qlb_check64_download", self._h, _lib.ptr(out), out.size)
        return out

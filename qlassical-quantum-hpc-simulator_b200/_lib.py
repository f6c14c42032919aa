"""ctypes binding of libqlassical_b200.so (the C ABI in include/qlassical_b200.h).

The library is built in-tree (``make -C qlassical-quantum-hpc-simulator_b200``)
and loaded from next to this file.  There is no fallback: if the shared
library is missing or cannot be loaded, importing the package raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqlassical_b200.so")

# ---------------------------------------------------------------------------
# Wire format: qlassical::GateInstr (frontend.hpp:84-105), 16 bytes.
# ---------------------------------------------------------------------------
GATE_INSTR_DTYPE = np.dtype(
    {
        "names": ["type", "flags_arity", "qubits", "qubits_ext", "payload", "uid"],
        "formats": ["u1", "u1", ("u1", (4,)), ("u1", (2,)), "<u4", "<u4"],
        "offsets": [0, 1, 2, 6, 8, 12],
        "itemsize": 16,
    }
)
MATRIX_ENTRY_DTYPE = np.dtype(
    {
        "names": ["offset", "num_elements", "num_qubits", "pad"],
        "formats": ["<u4", "<u4", "u1", ("u1", (3,))],
        "offsets": [0, 4, 8, 9],
        "itemsize": 12,
    }
)

QLB_OK = 0
QLB_ERR_INVALID_ARG = 1
QLB_ERR_OOM = 2
QLB_ERR_CUDA = 3
QLB_ERR_UNKNOWN_GATE = 4
QLB_ERR_NOT_NORMALIZED = 5
QLB_ERR_TIMEOUT = 6
QLB_ERR_STATE = 7

MODE_PLAIN = 0
MODE_TILED = 1
MODE_TILED_TC = 2

OPT_PHYSICAL_GLOBAL_SWAP = 1
OPT_TC_MIN_COST = 2
OPT_TC_CHAIN = 3
OPT_TILE_LOW = 4

BATCH_TUNE_CANDIDATES = 6
BATCH_TUNE_CLASSES = 18


class QlbError(RuntimeError):
    """A CUDA / device failure reported by the library."""


_EXC = {
    QLB_ERR_INVALID_ARG: ValueError,       # std::invalid_argument
    QLB_ERR_OOM: MemoryError,              # std::bad_alloc
    QLB_ERR_CUDA: QlbError,                # std::runtime_error
    QLB_ERR_UNKNOWN_GATE: RuntimeError,    # std::runtime_error (cpu_openmp_engine.hpp:221-222)
    QLB_ERR_NOT_NORMALIZED: ValueError,    # std::invalid_argument (cpu_state_vector.hpp:97-106)
    QLB_ERR_TIMEOUT: TimeoutError,
    QLB_ERR_STATE: RuntimeError,
}


class PoolView(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("num_elements", ctypes.c_uint64),
        ("metadata", ctypes.c_void_p),
        ("num_matrices", ctypes.c_uint64),
    ]


class ExecStats(ctypes.Structure):
    _fields_ = [
        ("instructions", ctypes.c_uint64),
        ("sweeps", ctypes.c_uint64),
        ("launches", ctypes.c_uint64),
        ("tile_passes", ctypes.c_uint64),
        ("permute_passes", ctypes.c_uint64),
        ("dense_ops", ctypes.c_uint64),
        ("tc_ops", ctypes.c_uint64),
        ("sweep_bytes", ctypes.c_double),
        ("chain_passes", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchTuneClass(ctypes.Structure):
    _fields_ = [
        ("num_qubits", ctypes.c_uint32),
        ("circuits", ctypes.c_uint32),
        ("sample", ctypes.c_uint32),
        ("best", ctypes.c_int32),
        ("ms", ctypes.c_float * BATCH_TUNE_CANDIDATES),
    ]


def batch_tune_candidate(i: int) -> dict:
    """Candidate i of the batched autotuner (qlb_batch_tune_class)."""
    return {"mode": "tiled" if i < 3 else "tiled_tc", "tile_low": 3 + i % 3}


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("circuits", ctypes.c_uint32),
        ("rounds", ctypes.c_uint32),
        ("mode", ctypes.c_int),
        ("launches", ctypes.c_uint32),
        ("tiles", ctypes.c_uint64),
        ("passes", ctypes.c_uint64),
        ("amp_updates", ctypes.c_uint64),
        ("state_bytes", ctypes.c_uint64),
        ("autotune_ms", ctypes.c_double * 2),
        ("tune_seconds", ctypes.c_double),
        ("tune_classes", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("tune", BatchTuneClass * BATCH_TUNE_CLASSES),
        ("fuse_seconds", ctypes.c_double),
        ("plan_seconds", ctypes.c_double),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [("memory_bytes", ctypes.c_uint64), ("mode", ctypes.c_int), ("max_active", ctypes.c_uint32),
                ("fuse_from", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class ServerInfo(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rounds", ctypes.c_uint64),
        ("launches", ctypes.c_uint64), ("tiles", ctypes.c_uint64), ("queued", ctypes.c_uint32),
        ("active", ctypes.c_uint32), ("arena_bytes", ctypes.c_uint64), ("arena_used", ctypes.c_uint64),
    ]


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("num_qubits", ctypes.c_uint32), ("passes", ctypes.c_uint32), ("shots", ctypes.c_uint64),
        ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
    ]


class Check64Result(ctypes.Structure):
    _fields_ = [("max_abs_diff", ctypes.c_double), ("infidelity", ctypes.c_double),
                ("norm_ref", ctypes.c_double), ("norm_state", ctypes.c_double),
                ("overlap_re", ctypes.c_double), ("overlap_im", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# qlb_cost_model_fn: (ctx, window_frequencies, log_to_phys, phys_to_log,
# num_qubits, *active, *victim) -> 1 to request a swap, 0 for none.
COST_MODEL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                 ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint16), ctypes.c_uint32,
                                 ctypes.POINTER(ctypes.c_uint16), ctypes.POINTER(ctypes.c_uint16))


class TranspileConfig(ctypes.Structure):
    _fields_ = [
        ("enable_gate_fusion", ctypes.c_int),
        ("enable_hw_awareness", ctypes.c_int),
        ("cost_model_type", ctypes.c_int),
        ("numa_penalty", ctypes.c_uint32),
        ("swap_penalty", ctypes.c_uint32),
        ("k_safe", ctypes.c_int),
        ("max_fusion_qubits", ctypes.c_int),
        ("reference_fusable_set", ctypes.c_int),
        ("custom_cost_model", COST_MODEL_FN),
        ("custom_cost_model_ctx", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I = ctypes.c_int
_PU64 = ctypes.POINTER(ctypes.c_uint64)
_PU32 = ctypes.POINTER(ctypes.c_uint32)
_PD = ctypes.POINTER(ctypes.c_double)

# name -> argtypes; every function returns int status (except the noted ones)
_SIGNATURES = {
    "qlb_set_device": [_I],
    "qlb_device_info": [ctypes.POINTER(ctypes.c_int), _PU64, _PU64],
    "qlb_selftest_bounded_wait": [_U32, ctypes.POINTER(ctypes.c_int)],
    "qlb_state_create": [ctypes.POINTER(_P)],
    "qlb_state_destroy": [_P],
    "qlb_state_initialize": [_P, _U32],
    "qlb_state_initialize_from": [_P, _P, _U64],
    "qlb_state_num_qubits": [_P, _PU32],
    "qlb_state_dimension": [_P, _PU64],
    "qlb_state_empty": [_P, ctypes.POINTER(ctypes.c_int)],
    "qlb_state_download": [_P, _P, _U64],
    "qlb_state_device_ptr": [_P, ctypes.POINTER(_P)],
    "qlb_engine_create": [ctypes.POINTER(_P), _U32, _I, _U64, _U64],
    "qlb_engine_create_from_amplitudes": [ctypes.POINTER(_P), _P, _U64, _I, _U64, _U64],
    "qlb_engine_create_from_state": [ctypes.POINTER(_P), _P],
    "qlb_engine_destroy": [_P],
    "qlb_engine_set_state_vector": [_P, _P],
    "qlb_engine_extract_state_vector": [_P, _P],
    "qlb_engine_reset": [_P],
    "qlb_engine_reset_to": [_P, _P, _U64],
    "qlb_engine_set_seed": [_P, _U64],
    "qlb_engine_reserve_measurements": [_P, _U64],
    "qlb_engine_measurements": [_P, ctypes.POINTER(_P), _PU64],
    "qlb_engine_execute": [_P, _P, _U64, ctypes.POINTER(PoolView)],
    "qlb_engine_state": [_P, _P, _U64],
    "qlb_engine_num_qubits": [_P, _PU32],
    "qlb_engine_set_mode": [_P, _I],
    "qlb_engine_get_mode": [_P, ctypes.POINTER(ctypes.c_int)],
    "qlb_engine_synchronize": [_P],
    "qlb_engine_device_state": [_P, ctypes.POINTER(_P)],
    "qlb_engine_stream": [_P, ctypes.POINTER(_P)],
    "qlb_engine_last_stats": [_P, ctypes.POINTER(ExecStats)],
    "qlb_engine_norm_sq": [_P, _PD],
    "qlb_engine_prob_one": [_P, _U32, _PD],
    "qlb_engine_expect_z": [_P, _P, _U32],
    "qlb_engine_sample": [_P, _U64, _U64, _P],
    "qlb_engine_amplitudes_at": [_P, _P, _U64, _P],
    "qlb_engine_set_option": [_P, _I, ctypes.c_int64],
    "qlb_engine_compile": [_P, _P, _U64, ctypes.POINTER(PoolView), ctypes.POINTER(_P)],
    "qlb_engine_run": [_P, _P],
    "qlb_plan_stats": [_P, ctypes.POINTER(ExecStats)],
    "qlb_plan_destroy": [_P],
    "qlb_check64_create": [ctypes.POINTER(_P), _U32],
    "qlb_check64_execute": [_P, _P, _U64, ctypes.POINTER(PoolView)],
    "qlb_check64_compare": [_P, _P, ctypes.POINTER(Check64Result)],
    "qlb_check64_download": [_P, _P, _U64],
    "qlb_check64_destroy": [_P],
    "qlb_batch_create": [ctypes.POINTER(_P), _U32, _P, _P, _P, _P, _I],
    "qlb_batch_create_ex": [ctypes.POINTER(_P), _U32, _P, _P, _P, _P, _I, _U32],
    "qlb_batch_run": [_P],
    "qlb_batch_synchronize": [_P],
    "qlb_batch_expect_z": [_P, _P, _U32],
    "qlb_batch_state": [_P, _U32, _P, _U64],
    "qlb_batch_stats": [_P, ctypes.POINTER(BatchInfo)],
    "qlb_batch_stream": [_P, ctypes.POINTER(_P)],
    "qlb_batch_destroy": [_P],
    "qlb_server_create": [ctypes.POINTER(_P), ctypes.POINTER(ServerConfig)],
    "qlb_server_submit": [_P, _P, _U64, ctypes.POINTER(PoolView), _U32, _U64, _U64, _PU64],
    "qlb_server_wait": [_P, _U64, ctypes.c_double],
    "qlb_server_result": [_P, _U64, _P, _U32, _P, _U64, ctypes.POINTER(RequestInfo)],
    "qlb_server_stats": [_P, ctypes.POINTER(ServerInfo)],
    "qlb_server_cancel": [_P, _U64],
    "qlb_server_destroy": [_P],
}
_OPTIONAL = {
    "qlb_transpile_gpu": [_P, _U64, ctypes.POINTER(PoolView), _U32, ctypes.POINTER(TranspileConfig),
                          ctypes.POINTER(_P)],
    "qlb_module_destroy": [_P],
    "qlb_module_program": [_P, ctypes.POINTER(_P), _PU64],
    "qlb_module_pool": [_P, ctypes.POINTER(PoolView)],
    "qlb_gpu_safe_qubit_limit": [_PU32],
}

_lib = None


def lib():
    """Loads (once) and returns the CDLL with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no CPU fallback exists)")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in {**_SIGNATURES, **_OPTIONAL}.items():
        if not hasattr(L, name):
            if name in _SIGNATURES:
                raise ImportError(f"{LIB_PATH} does not export {name}")
            continue
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.qlb_last_error.restype = ctypes.c_char_p
    L.qlb_last_error.argtypes = []
    L.qlb_version.restype = ctypes.c_char_p
    L.qlb_version.argtypes = []
    if hasattr(L, "qlb_transpile_config_default"):
        L.qlb_transpile_config_default.restype = None
        L.qlb_transpile_config_default.argtypes = [ctypes.POINTER(TranspileConfig)]
    _lib = L
    return L


def check(status: int) -> None:
    """Raises the Python counterpart of the reference's C++ exception."""
    if status == QLB_OK:
        return
    msg = lib().qlb_last_error().decode(errors="replace")
    raise _EXC.get(status, QlbError)(msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else 0

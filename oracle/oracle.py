"""TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU checkers.

  run_oracle(...)     the C restatement (sv_oracle.c), complex128
  run_reference(...)  the unmodified reference CPUOpenMPEngine (oracle/_ref)
  transpile_reference(...)  the reference Middleware::transpile (oracle/_ref)
  time_reference(...) the reference benchmark loop, for the CPU baseline

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libqlref.so")
REF_EXACT_SO = os.path.join(HERE, "_ref", "libqlref_exact.so")
# The reference source tree: $QLB_REFERENCE_DIR, else a directory named
# `reference` beside the repository (the layout this project is built in).
REFERENCE_DIR = os.environ.get(
    "QLB_REFERENCE_DIR", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


class _PoolView(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("num_elements", ctypes.c_uint64),
                ("metadata", ctypes.c_void_p), ("num_matrices", ctypes.c_uint64)]


def build(reference: bool | None = None) -> None:
    """Compiles the oracle (and, when the reference sources are present, the
    reference libraries) with oracle/Makefile."""
    targets = ["oracle"]
    if reference is None:
        reference = os.path.isdir(os.path.join(REFERENCE_DIR, "include"))
    if reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}"] + targets, check=True)


_libs: dict = {}


def _load(path: str):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing; run `make -C {HERE}`")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def reference_available() -> bool:
    return os.path.exists(REF_SO) and os.path.exists(REF_EXACT_SO)


def _pool_args(pool_data, pool_meta):
    data = np.ascontiguousarray(pool_data if pool_data is not None else np.zeros(0), dtype=np.complex128)
    meta = pool_meta
    if meta is None or len(meta) == 0:
        return _PoolView(None, 0, None, 0), (data, meta)
    meta = np.ascontiguousarray(meta)
    return _PoolView(data.ctypes.data if data.size else None, data.size, meta.ctypes.data, meta.size), (data, meta)


def _unpack_module(module):
    """(n, program, pool data, pool metadata) of an IR module, or of a
    ref_workloads.RefCircuit (numpy arrays only)."""
    if hasattr(module, "arrays"):
        n, prog, data, meta = module.arrays()
        return n, np.ascontiguousarray(prog), data, meta
    prog = np.ascontiguousarray(module.program())
    pool = module.unitaries()
    return module.num_qubits, prog, pool.data, pool.metadata()


def run_oracle(module, init=None, seed: int = 0, global_swap_noop: bool = False):
    """Returns (state complex128, measurements list)."""
    L = _load(ORACLE_SO)
    n, prog, pdata, pmeta = _unpack_module(module)
    pv, keep = _pool_args(pdata, pmeta)
    state = np.zeros(1 << n, dtype=np.complex128)
    if init is None:
        state[0] = 1.0
    else:
        state[:] = np.asarray(init, dtype=np.complex128)
    L.orc_rng_create.restype = ctypes.c_void_p
    L.orc_rng_create.argtypes = [ctypes.c_uint64]
    L.orc_rng_destroy.argtypes = [ctypes.c_void_p]
    L.orc_execute.restype = ctypes.c_int
    L.orc_execute.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64,
                              ctypes.POINTER(_PoolView), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                              ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint]
    rng = L.orc_rng_create(seed & 0xFFFFFFFFFFFFFFFF)
    meas = np.zeros(max(1, prog.size), dtype=np.uint8)
    cnt = ctypes.c_uint64(0)
    rc = L.orc_execute(state.ctypes.data, n, prog.ctypes.data if prog.size else None, prog.size,
                       ctypes.byref(pv), rng, meas.ctypes.data, meas.size, ctypes.byref(cnt),
                       1 if global_swap_noop else 0)
    L.orc_rng_destroy(rng)
    del keep
    if rc == -1:
        raise RuntimeError("oracle: Unrecognized instruction type")
    if rc != 0:
        raise ValueError("oracle: bad matrix index")
    return state, [int(x) for x in meas[:cnt.value]]


def run_reference(module, init=None, seed: int | None = 0, exact: bool = True):
    """Runs the unmodified reference engine; returns (state, measurements)."""
    L = _load(REF_EXACT_SO if exact else REF_SO)
    n, prog, pdata, pmeta = _unpack_module(module)
    pv, keep = _pool_args(pdata, pmeta)
    L.qlref_execute.restype = ctypes.c_int
    L.qlref_execute.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_PoolView),
                                ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    out = np.zeros(1 << n, dtype=np.complex128)
    ini = None if init is None else np.ascontiguousarray(init, dtype=np.complex128)
    meas = np.zeros(max(1, prog.size), dtype=np.uint8)
    cnt = ctypes.c_uint64(0)
    rc = L.qlref_execute(n, prog.ctypes.data if prog.size else None, prog.size, ctypes.byref(pv),
                         ini.ctypes.data if ini is not None else None, 0 if seed is None else 1,
                         0 if seed is None else seed, out.ctypes.data, meas.ctypes.data, meas.size,
                         ctypes.byref(cnt))
    del keep
    if rc == 4:
        raise RuntimeError("reference: Unrecognized instruction type")
    if rc == 1:
        raise ValueError("reference: invalid argument")
    if rc != 0:
        raise RuntimeError(f"reference failed ({rc})")
    return out, [int(x) for x in meas[:cnt.value]]


def transpile_reference(module, fusion=True, hw=False, cost_model=0, numa_penalty=10, swap_penalty=1,
                        k_safe=-1):
    """Reference Middleware::transpile(module, CPU_OPENMP, cfg); returns
    (program array, pool data, pool metadata)."""
    from importlib import import_module  # noqa: F401  (keeps module import-light)
    L = _load(REF_EXACT_SO)
    n, prog, pdata, pmeta = _unpack_module(module)
    pv, keep = _pool_args(pdata, pmeta)
    L.qlref_transpile.restype = ctypes.c_void_p
    L.qlref_transpile.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_PoolView),
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_int]
    for f in ("qlref_module_count", "qlref_module_pool_elements", "qlref_module_pool_matrices"):
        getattr(L, f).restype = ctypes.c_uint64
        getattr(L, f).argtypes = [ctypes.c_void_p]
    L.qlref_module_copy.argtypes = [ctypes.c_void_p] * 4
    L.qlref_module_free.argtypes = [ctypes.c_void_p]
    h = L.qlref_transpile(n, prog.ctypes.data if prog.size else None, prog.size, ctypes.byref(pv),
                          int(fusion), int(hw), int(cost_model), numa_penalty, swap_penalty, k_safe)
    del keep
    if not h:
        raise ValueError("reference transpile failed")
    cnt = L.qlref_module_count(h)
    ne = L.qlref_module_pool_elements(h)
    nm = L.qlref_module_pool_matrices(h)
    from . import ref_workloads
    out = np.zeros(cnt, dtype=prog.dtype)
    data = np.zeros(ne, dtype=np.complex128)
    meta = np.zeros(nm, dtype=pmeta.dtype if pmeta is not None else ref_workloads.MATRIX_ENTRY_DTYPE)
    L.qlref_module_copy(h, out.ctypes.data if cnt else None, data.ctypes.data if ne else None,
                        meta.ctypes.data if nm else None)
    L.qlref_module_free(h)
    return out, data, meta


def time_reference(module, reps: int = 1) -> float:
    """Mean wall seconds of the reference execute() (Release build)."""
    L = _load(REF_SO)
    n, prog, pdata, pmeta = _unpack_module(module)
    pv, keep = _pool_args(pdata, pmeta)
    L.qlref_time_execute.restype = ctypes.c_double
    L.qlref_time_execute.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(_PoolView),
                                     ctypes.c_int]
    t = L.qlref_time_execute(n, prog.ctypes.data if prog.size else None, prog.size, ctypes.byref(pv), reps)
    del keep
    return t


def reference_threads() -> int:
    L = _load(REF_SO)
    L.qlref_num_threads.restype = ctypes.c_int
    return L.qlref_num_threads()


def infidelity(a: np.ndarray, b: np.ndarray) -> float:
    """1 - |<a|b>|^2 / (<a|a><b|b>), computed in float64."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    ov = np.vdot(a, b)
    return float(1.0 - (abs(ov) ** 2) / (np.vdot(a, a).real * np.vdot(b, b).real))


def max_abs_diff(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(a) else 0.0

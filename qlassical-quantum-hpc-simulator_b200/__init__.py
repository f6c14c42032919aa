"""Qlassical B200 backend: a CUDAEngine / CUDAStateVector for the Qlassical
state-vector simulator, implemented as hand-written sm_100a CUDA kernels
behind a C ABI (include/qlassical_b200.h).  This Python package is the
host-side mirror of the reference's frontend / backend interfaces used by
the tests and the benchmark; the C++20 drop-in lives in
include/qlassical_b200/.
"""
from . import _lib
from ._lib import QlbError, lib
from .ir import GateType, IRModule, QuantumCircuit, UnitaryPool, make_instr
from .engine import Check64, CUDAEngine, CUDAStateVector

lib()  # fail loudly at import if the native library is missing

__all__ = [
    "GateType", "IRModule", "QuantumCircuit", "UnitaryPool", "make_instr",
    "CUDAEngine", "CUDAStateVector", "Check64", "QlbError", "lib",
]

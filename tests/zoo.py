"""Seeded random circuits over every instruction type, for parity tests."""
from __future__ import annotations

import math

import numpy as np

from qlassical_b200.ir import GateType, IRModule, QuantumCircuit, UnitaryPool, make_instr


def random_unitary(k: int, rng: np.random.Generator) -> np.ndarray:
    d = 1 << k
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / math.sqrt(2.0)
    q, r = np.linalg.qr(z)
    ph = np.diag(r) / np.abs(np.diag(r))
    return q * ph


REF_TYPES = ["h", "x", "y", "z", "s", "rx", "ry", "rz", "cx", "swap", "ccx", "cswap", "u1", "u2", "u3", "u4",
             "barrier"]
EXT_TYPES = ["cz", "cp", "u5", "u6", "diag1", "diag2"]


def random_circuit(n: int, count: int, seed: int, types=None, max_dense: int = 4) -> IRModule:
    """`count` instructions drawn uniformly from `types` on random qubits."""
    rng = np.random.default_rng(seed)
    types = list(types or REF_TYPES)
    types = [t for t in types if not (t.startswith("u") and int(t[1:]) > min(max_dense, n))]
    if n < 3:
        types = [t for t in types if t not in ("ccx", "cswap")]
    if n < 2:
        types = [t for t in types if t not in ("cx", "swap", "cz", "cp", "diag2")]
    qc = QuantumCircuit(n)
    for _ in range(count):
        t = types[rng.integers(len(types))]
        qs = [int(v) for v in rng.permutation(n)[:6]]
        th = float(rng.uniform(0, 2 * math.pi))
        if t in ("h", "x", "y", "z", "s"):
            getattr(qc, t)(qs[0])
        elif t in ("rx", "ry", "rz"):
            getattr(qc, t)(qs[0], th)
        elif t in ("cx", "swap", "cz"):
            getattr(qc, t)(qs[0], qs[1])
        elif t == "cp":
            qc.cp(qs[0], qs[1], th)
        elif t in ("ccx", "cswap"):
            getattr(qc, t)(qs[0], qs[1], qs[2])
        elif t.startswith("u"):
            k = int(t[1:])
            qc.unitary(qs[:k], random_unitary(k, rng))
        elif t == "diag1":
            qc.unitary(qs[:1], np.diag(np.exp(1j * rng.uniform(0, 2 * math.pi, 2))))
        elif t == "diag2":
            qc.unitary(qs[:2], np.diag(np.exp(1j * rng.uniform(0, 2 * math.pi, 4))))
        elif t == "barrier":
            qc.barrier(qs[:2])
    return qc.release()


def random_state(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def module_from_arrays(n: int, prog: np.ndarray, pool_data: np.ndarray, pool_meta: np.ndarray) -> IRModule:
    m = IRModule(n, unitary_pool=UnitaryPool.from_arrays(pool_data, pool_meta))
    m.set_program(prog)
    return m

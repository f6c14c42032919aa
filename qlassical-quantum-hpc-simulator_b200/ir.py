"""IR types and circuit builder, mirroring Qlassical's frontend
(include/frontend/frontend.hpp): GateType (:26-51), GateInstr (:84-105),
UnitaryPool (:117-164), IRModule (:172-201) and the QuantumCircuit builder
(:218-497) with the same method names, argument meaning and errors
(std::out_of_range -> IndexError, std::invalid_argument -> ValueError).

Additive extensions (absent from the reference, which expresses them as
2-qubit UNITARY diagonals): ``cz`` and ``cp`` gate types, and dense blocks
of 5-6 qubits whose qubits 4 and 5 ride in the instruction's two pad bytes.
"""
from __future__ import annotations

import enum
from typing import Iterable, Sequence

import numpy as np

from ._lib import GATE_INSTR_DTYPE, MATRIX_ENTRY_DTYPE, PoolView

NO_MATRIX = 0xFFFFFFFF


class GateType(enum.IntEnum):
    H = 0x00
    X = 0x01
    Y = 0x02
    Z = 0x03
    S = 0x04
    RX = 0x10
    RY = 0x11
    RZ = 0x12
    CX = 0x20
    SWAP = 0x21
    CZ = 0x22       # additive
    CP = 0x23       # additive, payload.param = phi
    CCX = 0x30
    CSWAP = 0x31
    UNITARY = 0x80
    FUSED_BLOCK = 0xE0
    GLOBAL_SWAP = 0xE1
    BARRIER = 0xF0
    MEASURE = 0xF1


def gate_arity(t: int) -> int:
    """frontend.hpp:504-512."""
    if t < 0x20:
        return 1
    if t < 0x30:
        return 2
    if t < 0x40:
        return 3
    return 0


def gate_is_parametric(t: int) -> bool:
    """frontend.hpp:515-518 (CP, additive, also carries a parameter)."""
    return 0x10 <= t < 0x20


def gate_uses_matrix(t: int) -> bool:
    return t in (GateType.UNITARY, GateType.FUSED_BLOCK)


def gate_is_directive(t: int) -> bool:
    return t >= 0xE0


def f32_bits(x: float) -> int:
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])


def bits_f32(u: int) -> float:
    return float(np.array([u], dtype=np.uint32).view(np.float32)[0])


def make_instr(gtype: int, qubits: Sequence[int] = (), param: float = 0.0, matrix_idx: int | None = None,
               uid: int = 0, flags: int = 0) -> np.void:
    """One GateInstr record (the `make_gate` helper of the reference tests)."""
    rec = np.zeros(1, dtype=GATE_INSTR_DTYPE)[0]
    rec["type"] = int(gtype)
    k = len(qubits)
    rec["flags_arity"] = (k & 0x0F) | ((flags & 0x0F) << 4)
    q = [255, 255, 255, 255]
    ext = [0, 0]
    for j, v in enumerate(qubits):
        if j < 4:
            q[j] = int(v)
        else:
            ext[j - 4] = int(v)
    rec["qubits"] = q
    rec["qubits_ext"] = ext
    rec["payload"] = int(matrix_idx) if matrix_idx is not None else f32_bits(param)
    rec["uid"] = uid
    return rec


class UnitaryPool:
    """Flat row-major complex128 storage + per-matrix metadata."""

    def __init__(self):
        self._chunks: list[np.ndarray] = []
        self._meta: list[tuple[int, int, int]] = []
        self._size = 0
        self._cache = None

    def store(self, matrix, num_qubits: int) -> int:
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(-1))
        expected = 1 << (2 * num_qubits)
        if m.size != expected:
            raise ValueError(
                f"UnitaryPool::store: matrix size mismatch. Expected {expected}, got {m.size}")
        idx = len(self._meta)
        self._meta.append((self._size, expected, num_qubits))
        self._chunks.append(m)
        self._size += expected
        self._cache = None
        return idx

    def get(self, idx: int) -> np.ndarray:
        off, n, k = self._meta[idx]
        d = 1 << k
        return self.data[off:off + n].reshape(d, d)

    def num_matrices(self) -> int:
        return len(self._meta)

    def total_elements(self) -> int:
        return self._size

    def empty(self) -> bool:
        return not self._meta

    @property
    def data(self) -> np.ndarray:
        if self._cache is None:
            self._cache = (np.concatenate(self._chunks) if self._chunks
                           else np.zeros(0, dtype=np.complex128))
        return self._cache

    def metadata(self) -> np.ndarray:
        meta = np.zeros(len(self._meta), dtype=MATRIX_ENTRY_DTYPE)
        for i, (off, n, k) in enumerate(self._meta):
            meta[i]["offset"] = off
            meta[i]["num_elements"] = n
            meta[i]["num_qubits"] = k
        return meta

    @classmethod
    def from_arrays(cls, data: np.ndarray, meta: np.ndarray) -> "UnitaryPool":
        p = cls()
        data = np.asarray(data, dtype=np.complex128)
        for e in meta:
            off, n, k = int(e["offset"]), int(e["num_elements"]), int(e["num_qubits"])
            p.store(data[off:off + n], k)
        return p

    def view(self):
        """A qlb_pool_view over this pool; keep the returned tuple alive."""
        data = np.ascontiguousarray(self.data)
        meta = self.metadata()
        pv = PoolView(data.ctypes.data if data.size else None, data.size,
                      meta.ctypes.data if meta.size else None, meta.size)
        return pv, (data, meta)


class IRModule:
    """Move-only in the reference; here a plain container."""

    def __init__(self, num_qubits: int = 0, gate_stream=None, unitary_pool: UnitaryPool | None = None):
        self.num_qubits = int(num_qubits)
        self._gates: list = list(gate_stream) if gate_stream is not None else []
        self.unitary_pool = unitary_pool if unitary_pool is not None else UnitaryPool()

    def program(self) -> np.ndarray:
        """The gate stream as one contiguous GateInstr array (the reference
        keeps gate_stream contiguous).  Records appended one at a time are
        packed on the first call and the packed array is kept until the next
        append."""
        if not isinstance(self._gates, np.ndarray):
            self._gates = (np.array(self._gates, dtype=GATE_INSTR_DTYPE) if self._gates
                           else np.zeros(0, dtype=GATE_INSTR_DTYPE))
        return self._gates

    def set_program(self, arr: np.ndarray) -> None:
        self._gates = np.ascontiguousarray(arr, dtype=GATE_INSTR_DTYPE)

    def append(self, rec) -> None:
        if isinstance(self._gates, np.ndarray):
            self._gates = list(self._gates)
        self._gates.append(rec)

    def unitaries(self) -> UnitaryPool:
        return self.unitary_pool

    def gate_count(self) -> int:
        return len(self._gates)

    def empty(self) -> bool:
        return len(self._gates) == 0


class QuantumCircuit:
    """Fluent builder (frontend.hpp:218-497)."""

    def __init__(self, num_qubits: int, gate_count_hint: int = 256):
        self._module = IRModule(num_qubits)
        self._uid = 0

    def release(self) -> IRModule:
        m = self._module
        self._module = IRModule(m.num_qubits)
        return m

    def num_qubits(self) -> int:
        return self._module.num_qubits

    def size(self) -> int:
        return self._module.gate_count()

    def program(self) -> np.ndarray:
        return self._module.program()

    # -- validation (frontend.hpp:410-416, 449-452, 466-468) ---------------
    def _validate(self, q: int) -> None:
        if q < 0 or q >= 256 or q >= self._module.num_qubits:
            raise IndexError(
                f"Qubit index {q} out of range [0, min(256, {self._module.num_qubits}))")

    def _push(self, gtype, qubits, param=0.0, matrix_idx=None):
        for q in qubits:
            self._validate(q)
        if len(set(qubits)) != len(qubits):
            if len(qubits) == 2:
                raise ValueError(f"Two-qubit gate requires distinct qubits, got {qubits[0]} == {qubits[1]}")
            raise ValueError("Three-qubit gate requires distinct qubits")
        self._module.append(make_instr(gtype, qubits, param, matrix_idx, uid=self._uid))
        self._uid += 1
        return self

    def h(self, q): return self._push(GateType.H, [q])
    def x(self, q): return self._push(GateType.X, [q])
    def y(self, q): return self._push(GateType.Y, [q])
    def z(self, q): return self._push(GateType.Z, [q])
    def s(self, q): return self._push(GateType.S, [q])
    def rx(self, q, theta): return self._push(GateType.RX, [q], float(np.float32(theta)))
    def ry(self, q, theta): return self._push(GateType.RY, [q], float(np.float32(theta)))
    def rz(self, q, theta): return self._push(GateType.RZ, [q], float(np.float32(theta)))
    def cx(self, c, t): return self._push(GateType.CX, [c, t])
    cnot = cx
    def swap(self, a, b): return self._push(GateType.SWAP, [a, b])
    def cz(self, a, b): return self._push(GateType.CZ, [a, b])
    def cp(self, a, b, phi): return self._push(GateType.CP, [a, b], float(np.float32(phi)))
    def ccx(self, c0, c1, t): return self._push(GateType.CCX, [c0, c1, t])
    toffoli = ccx
    def cswap(self, c, a, b): return self._push(GateType.CSWAP, [c, a, b])
    fredkin = cswap

    def unitary(self, target_qubits: Sequence[int], matrix) -> "QuantumCircuit":
        k = len(target_qubits)
        if k == 0 or k > 6:
            raise ValueError(f"unitary: arity must be 1-6, got {k}")
        for q in target_qubits:
            self._validate(q)
        if len(set(target_qubits)) != k:
            raise ValueError("unitary: qubits must be distinct")
        midx = self._module.unitary_pool.store(matrix, k)
        self._module.append(make_instr(GateType.UNITARY, list(target_qubits), matrix_idx=midx, uid=self._uid))
        self._uid += 1
        return self

    def barrier(self, qubits: Iterable[int] = ()) -> "QuantumCircuit":
        qs = list(qubits)[:4]
        for q in qs:
            self._validate(q)
        self._module.append(make_instr(GateType.BARRIER, qs, uid=self._uid))
        self._uid += 1
        return self

    def measure(self, q) -> "QuantumCircuit":
        if isinstance(q, (list, tuple)):
            for v in q:
                self.measure(v)
            return self
        return self._push(GateType.MEASURE, [q])

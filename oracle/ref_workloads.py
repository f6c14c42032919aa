"""TEST INFRASTRUCTURE ONLY -- the benchmark circuits in the reference's own
IR, built with numpy alone (no import of the package under test), for the
reference arm of bench.py and the CPU baseline.

The records are qlassical::GateInstr (frontend.hpp:84-105: type, arity,
qubits[4] with 255 for unused slots, two pad bytes, a float angle or a
matrix index, uid) and the pool is UnitaryPool (frontend.hpp:117-164:
complex128 row-major data plus 12-byte MatrixEntry records).  The reference
has no CZ gate type, so CZ is the 2-qubit UNITARY diag(1, 1, 1, -1), stored
once in the pool, which is how its own tests express it.  The draws follow
the package's circuit generators exactly (numpy PCG64 seeded with `seed`,
angles rounded to float32 as the reference builder stores them,
frontend.hpp:280-292); tests/test_oracle_pinning.py checks the bytes.
"""
from __future__ import annotations

import math

import numpy as np

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

RX, RY, RZ, UNITARY = 0x10, 0x11, 0x12, 0x80


class RefCircuit:
    """A program in the reference IR: `num_qubits`, `prog` (GateInstr
    records), `pool_data` (complex128) and `pool_meta` (MatrixEntry)."""

    def __init__(self, num_qubits, prog, pool_data, pool_meta, layer_starts=None):
        self.num_qubits = int(num_qubits)
        self.prog = prog
        self.pool_data = pool_data
        self.pool_meta = pool_meta
        self.layer_starts = layer_starts or [0]

    def arrays(self):
        return self.num_qubits, self.prog, self.pool_data, self.pool_meta

    def gate_count(self) -> int:
        return int(self.prog.size)

    def layers(self, first: int, count: int) -> "RefCircuit":
        """Whole layers [first, first + count) with the same pool."""
        starts = self.layer_starts + [self.prog.size]
        lo, hi = starts[first], starts[min(first + count, len(self.layer_starts))]
        return RefCircuit(self.num_qubits, self.prog[lo:hi].copy(), self.pool_data, self.pool_meta,
                          [s - lo for s in self.layer_starts[first:first + count]])


def _f32_bits(x: float) -> int:
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])


def random_rot_cz(n: int = 30, depth: int = 24, seed: int = 1234) -> RefCircuit:
    """Per layer: RX/RY/RZ(theta~U[0,2pi)) on every qubit (type drawn from
    the seeded stream), then CZ on seeded random disjoint pairs covering the
    full qubit range, as 2-qubit UNITARY diagonals."""
    rng = np.random.default_rng(seed)
    records = []
    starts = []
    uid = 0
    for _ in range(depth):
        starts.append(len(records))
        kinds = rng.integers(0, 3, size=n)
        thetas = rng.uniform(0.0, 2.0 * math.pi, size=n)
        for q in range(n):
            records.append(((RX, RY, RZ)[kinds[q]], 1, (q, 255, 255, 255), _f32_bits(float(np.float32(thetas[q]))),
                            uid))
            uid += 1
        perm = rng.permutation(n)
        for i in range(0, n - 1, 2):
            records.append((UNITARY, 2, (int(perm[i]), int(perm[i + 1]), 255, 255), 0, uid))
            uid += 1
    prog = np.zeros(len(records), dtype=GATE_INSTR_DTYPE)
    for i, (t, k, qs, payload, u) in enumerate(records):
        prog[i]["type"] = t
        prog[i]["flags_arity"] = k
        prog[i]["qubits"] = qs
        prog[i]["payload"] = payload
        prog[i]["uid"] = u
    data = np.diag(np.array([1.0, 1.0, 1.0, -1.0], dtype=np.complex128)).reshape(-1)
    meta = np.zeros(1, dtype=MATRIX_ENTRY_DTYPE)
    meta[0]["offset"] = 0
    meta[0]["num_elements"] = 16
    meta[0]["num_qubits"] = 2
    return RefCircuit(n, prog, data, meta, starts)


H, SWAP = 0x00, 0x21


def qft(n: int) -> RefCircuit:
    """QFT|0...0> in the reference IR: for i = n-1 .. 0, H(i) then CP(j, i,
    pi/2^(i-j)) for j = i-1 .. 0 as 2-qubit UNITARY diag(1, 1, 1, e^{i phi})
    (phi rounded to float32 as the IR stores angles; one pool matrix per
    distinct angle, in order of first use); finally SWAP(i, n-1-i)."""
    records = []
    mats = []
    index = {}
    uid = 0
    for i in range(n - 1, -1, -1):
        records.append((H, 1, (i, 255, 255, 255), 0, uid))
        uid += 1
        for j in range(i - 1, -1, -1):
            bits = _f32_bits(math.pi / float(1 << (i - j)))
            if bits not in index:
                phi = float(np.array([bits], dtype=np.uint32).view(np.float32)[0])
                index[bits] = len(mats)
                mats.append(np.diag(np.array([1.0, 1.0, 1.0, complex(math.cos(phi), math.sin(phi))],
                                             dtype=np.complex128)).reshape(-1))
            records.append((UNITARY, 2, (j, i, 255, 255), index[bits], uid))
            uid += 1
    for i in range(n // 2):
        records.append((SWAP, 2, (i, n - 1 - i, 255, 255), 0, uid))
        uid += 1
    prog = np.zeros(len(records), dtype=GATE_INSTR_DTYPE)
    for r, (t, k, qs, payload, u) in enumerate(records):
        prog[r]["type"] = t
        prog[r]["flags_arity"] = k
        prog[r]["qubits"] = qs
        prog[r]["payload"] = payload
        prog[r]["uid"] = u
    data = np.concatenate(mats) if mats else np.zeros(0, dtype=np.complex128)
    meta = np.zeros(len(mats), dtype=MATRIX_ENTRY_DTYPE)
    for i in range(len(mats)):
        meta[i]["offset"] = 16 * i
        meta[i]["num_elements"] = 16
        meta[i]["num_qubits"] = 2
    return RefCircuit(n, prog, data, meta)

"""CPU-only checks of the boundary: the C-ABI library loads and exports every
function include/*.h declares, the wire format matches the reference's
GateInstr layout, and the host-side builder / generators behave like the
reference's (no GPU needed; no compute calls)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import _lib, circuits
from qlassical_b200.ir import GateType, QuantumCircuit, UnitaryPool

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(qlb_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "qlb_engine_execute" in names and len(names) > 30


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    assert hasattr(_lib.lib(), name), f"{name} declared in include/*.h but not exported"


def test_gate_instr_layout_matches_reference():
    """test_frontend.cpp:26-37: 16 bytes, offsets 0/1/2/8/12."""
    d = _lib.GATE_INSTR_DTYPE
    assert d.itemsize == 16
    assert d.fields["type"][1] == 0 and d.fields["flags_arity"][1] == 1
    assert d.fields["qubits"][1] == 2 and d.fields["payload"][1] == 8 and d.fields["uid"][1] == 12
    assert _lib.MATRIX_ENTRY_DTYPE.itemsize == 12


def test_builder_validation_errors():
    """frontend.hpp:410-416, 449-452, 466-468, 343-346."""
    qc = QuantumCircuit(3)
    with pytest.raises(IndexError):
        qc.h(3)
    with pytest.raises(IndexError):
        qc.x(-1)
    with pytest.raises(ValueError):
        qc.cx(1, 1)
    with pytest.raises(ValueError):
        qc.ccx(0, 1, 1)
    with pytest.raises(ValueError):
        qc.unitary([], np.eye(1))
    with pytest.raises(ValueError):
        UnitaryPool().store(np.eye(3), 1)


def test_builder_records_float_params_and_uids():
    qc = QuantumCircuit(2)
    qc.rx(0, 0.1).cx(0, 1).measure([0, 1])
    p = qc.program()
    assert list(p["uid"]) == [0, 1, 2, 3]
    assert p[0]["flags_arity"] & 0xF == 1
    assert abs(np.array([p[0]["payload"]], dtype=np.uint32).view(np.float32)[0] - np.float32(0.1)) == 0
    assert p[1]["type"] == GateType.CX and list(p[1]["qubits"][:2]) == [0, 1]


def test_wide_unitary_uses_pad_bytes():
    qc = QuantumCircuit(8)
    qc.unitary([0, 1, 2, 3, 6, 7], np.eye(64))
    rec = qc.program()[0]
    assert rec["flags_arity"] & 0xF == 6
    assert list(rec["qubits"]) == [0, 1, 2, 3] and list(rec["qubits_ext"]) == [6, 7]


def test_workload_shapes():
    m0 = circuits.random_h_rx_cx(20, 40, seed=1)
    assert m0.gate_count() == 40 * 20 + 20 * 19   # 1180 (survey-time probe count)
    m1 = circuits.random_rot_cz(30, 24, seed=1)
    assert m1.gate_count() == 24 * (30 + 15)
    m2 = circuits.qft(33)
    assert m2.gate_count() == 33 + 33 * 32 // 2 + 16
    assert circuits.clustered(28).gate_count() == 765   # bench.txt:9


def test_reference_ir_rewrites_cz_cp():
    m = circuits.random_rot_cz(6, 2, seed=3)
    r = circuits.to_reference_ir(m)
    t = r.program()["type"]
    assert not np.any((t == GateType.CZ) | (t == GateType.CP))
    assert np.count_nonzero(t == GateType.UNITARY) == 2 * 3


def test_no_device_fails_loudly():
    """Without a GPU the engine raises instead of computing on the CPU."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    with pytest.raises((q.QlbError, MemoryError, RuntimeError)):
        q.CUDAEngine(4)

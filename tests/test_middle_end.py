"""The GPU middle end (transpile_gpu) on the CPU: restated middleware KATs
(tests/middleware/test_middleware.cpp, test_fusion_math.cpp), parity of
the fusion pass with the reference's at k <= 4 (oracle/_ref), and the
numerical equivalence of every transpiled stream with its input (the
check the reference never makes, SURVEY gap: windowing corrupts states)."""
import numpy as np
import pytest

from qlassical_b200 import circuits
from qlassical_b200.ir import GateType, QuantumCircuit
from qlassical_b200.middleware import (Backend, CostModelType, Middleware, TranspilerConfig, WindowingCostModel,
                                       gpu_safe_qubit_limit)
from oracle import oracle
import zoo


def tp(module, **kw):
    return Middleware().transpile(module, Backend.GPU, TranspilerConfig(**kw))


def test_config_defaults():
    """test_middleware.cpp:142-162."""
    c = TranspilerConfig()
    assert c.enable_gate_fusion and c.enable_hw_awareness
    assert c.cost_model_type == CostModelType.THRESHOLD
    assert c.numa_penalty == 10 and c.swap_penalty == 1 and c.k_safe is None and c.custom_cost_model is None


def test_gpu_topology_window():
    assert gpu_safe_qubit_limit() == 13


def test_fusion_heuristic_kats():
    """test_middleware.cpp:60-92."""
    qc = QuantumCircuit(2)
    qc.h(0).x(1)
    out = tp(qc.release(), enable_hw_awareness=False, max_fusion_qubits=4, reference_fusable_set=True)
    assert [int(t) for t in out.program()["type"]] == [GateType.H, GateType.X]
    qc = QuantumCircuit(2)
    qc.h(0).cx(0, 1).x(1)
    out = tp(qc.release(), enable_hw_awareness=False, max_fusion_qubits=4, reference_fusable_set=True)
    p = out.program()
    assert len(p) == 1 and p[0]["type"] == GateType.FUSED_BLOCK and p[0]["flags_arity"] & 0xF == 2


def test_fusion_math_kats():
    """test_fusion_math.cpp:17-150 through one fused block: X then Z on q0
    gives Z*X; CX(0,1) then CZ(1,2) gives entries (1,3), (5,7), (7,5)."""
    qc = QuantumCircuit(1)
    sx = np.array([[0, 1], [1, 0]], dtype=complex)
    sz = np.array([[1, 0], [0, -1]], dtype=complex)
    qc.unitary([0], sx).unitary([0], sz)
    out = tp(qc.release(), enable_hw_awareness=False)
    assert np.allclose(out.unitaries().get(int(out.program()[0]["payload"])), sz @ sx)
    qc = QuantumCircuit(3)
    cx = np.eye(4, dtype=complex)[[0, 3, 2, 1]]
    cz = np.diag([1, 1, 1, -1]).astype(complex)
    qc.unitary([0, 1], cx).unitary([1, 2], cz)
    out = tp(qc.release(), enable_hw_awareness=False)
    p = out.program()
    assert len(p) == 1 and list(p[0]["qubits"][:3]) == [0, 1, 2]
    f = out.unitaries().get(int(p[0]["payload"]))
    assert abs(f[1, 3] - 1) < 1e-12 and abs(f[5, 7] - 1) < 1e-12 and abs(f[7, 5] + 1) < 1e-12


def _tlb_module():
    qc = QuantumCircuit(10)
    qc.x(0).x(1).cx(8, 9)
    return qc.release()


def test_windowing_tlb_hazard():
    """test_middleware.cpp:94-140 (ThresholdCostModel(2, 1, 0))."""
    out = tp(_tlb_module(), enable_gate_fusion=False, k_safe=2, numa_penalty=1, swap_penalty=0)
    p = out.program()
    assert len(p) == 5
    assert [int(t) for t in p["type"][:2]] == [GateType.X, GateType.X]
    assert p[2]["type"] == GateType.GLOBAL_SWAP and p[3]["type"] == GateType.GLOBAL_SWAP
    assert p[2]["qubits"][0] in (8, 9) and p[2]["qubits"][1] in (0, 1)
    assert p[2]["qubits"][0] != p[3]["qubits"][0] and p[2]["qubits"][1] != p[3]["qubits"][1]
    assert p[4]["type"] == GateType.CX and set(p[4]["qubits"][:2]) == {0, 1}


def test_windowing_penalties_and_greedy():
    """test_middleware.cpp:164-235."""
    out = tp(_tlb_module(), enable_gate_fusion=False, k_safe=2, numa_penalty=1, swap_penalty=100)
    assert out.gate_count() == 3 and list(out.program()[2]["qubits"][:2]) == [8, 9]
    out = tp(_tlb_module(), enable_gate_fusion=False, k_safe=2, numa_penalty=10, swap_penalty=1)
    assert out.gate_count() == 5
    out = tp(_tlb_module(), enable_gate_fusion=False, k_safe=2, cost_model_type=CostModelType.GREEDY)
    assert out.gate_count() == 5
    out = tp(_tlb_module(), enable_gate_fusion=False, k_safe=16)
    assert out.gate_count() == 3


class Spy(WindowingCostModel):
    def __init__(self):
        self.evaluated = False

    def get_k_safe(self):
        return 3

    def evaluate_swap(self, f, l2p, p2l):
        self.evaluated = True
        return None


def test_custom_cost_model_hook():
    """test_middleware.cpp:237-294."""
    qc = QuantumCircuit(6)
    qc.h(0).cx(4, 5)
    spy = Spy()
    cfg = TranspilerConfig(enable_gate_fusion=False)
    cfg.set_cost_model(spy)
    out = Middleware().transpile(qc.release(), Backend.GPU, cfg)
    assert spy.evaluated and out.gate_count() == 2
    qc = QuantumCircuit(4)
    qc.h(0)
    with pytest.raises(ValueError):
        Middleware().transpile(qc.release(), Backend.GPU, TranspilerConfig(cost_model_type=CostModelType.CUSTOM))


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", range(5))
def test_fusion_matches_reference_at_k4(seed):
    """With the reference's limits (k <= 4, its fusable set) the GPU fusion
    pass emits the reference's stream and matrices."""
    m = zoo.random_circuit(9, 120, seed=300 + seed, types=["h", "x", "y", "z", "s", "cx", "u1", "u2", "rx", "ccx"])
    prog, data, meta = oracle.transpile_reference(m, fusion=True, hw=False)
    out = tp(m, enable_hw_awareness=False, max_fusion_qubits=4, reference_fusable_set=True)
    op = out.program()
    assert len(op) == len(prog)
    assert np.array_equal(op["type"], prog["type"])
    assert np.array_equal(op["qubits"], prog["qubits"]) and np.array_equal(op["flags_arity"], prog["flags_arity"])
    for g, r in zip(op, prog):
        if g["type"] == GateType.FUSED_BLOCK:
            a = out.unitaries().get(int(g["payload"]))
            k = int(r["flags_arity"]) & 0xF
            e = meta[int(r["payload"])]
            b = data[int(e["offset"]):int(e["offset"]) + int(e["num_elements"])].reshape(1 << k, 1 << k)
            assert np.max(np.abs(a - b)) < 1e-12


@pytest.mark.parametrize("kmax", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("windowing", [False, True])
def test_transpiled_stream_is_equivalent(kmax, windowing):
    m = zoo.random_circuit(12, 160, seed=kmax, types=zoo.REF_TYPES + ["cz", "cp", "diag2"])
    want, _ = oracle.run_oracle(m)
    out = tp(m, max_fusion_qubits=kmax, enable_hw_awareness=windowing, k_safe=5)
    got, _ = oracle.run_oracle(out)
    assert oracle.max_abs_diff(want, got) < 1e-10
    assert out.gate_count() <= m.gate_count() + (200 if windowing else 0)


def test_config1_recipe_fuses_to_five_qubit_blocks():
    m = circuits.random_rot_cz(14, 6, seed=9)
    out = tp(m, enable_hw_awareness=False, max_fusion_qubits=5)
    ar = out.program()["flags_arity"] & 0xF
    assert ar.max() <= 5 and out.gate_count() < m.gate_count() // 3
    want, _ = oracle.run_oracle(m)
    got, _ = oracle.run_oracle(out)
    assert oracle.max_abs_diff(want, got) < 1e-10

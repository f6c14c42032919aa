"""GPU parity: CUDAEngine (through the C ABI) against the oracle and the
reference fixtures.  Tolerances (complex64 state, FP32 arithmetic):
max |delta amplitude| <= 2e-5 and infidelity 1 - |<ref|psi>|^2 <= 1e-6."""
import math

import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import circuits
from qlassical_b200.ir import GateType, IRModule, QuantumCircuit, make_instr
from golden_cases import load_cases
from oracle import oracle
import zoo

pytestmark = pytest.mark.gpu

MAX_DIFF = 2e-5
MAX_INFID = 1e-6
MODES = ["plain", "tiled", "tiled_tc"]
CASES = load_cases()


def check_close(ref, got, tol=MAX_DIFF, infid=MAX_INFID):
    d = oracle.max_abs_diff(ref, got)
    f = oracle.infidelity(ref, got)
    assert d <= tol and f <= infid, f"max|d|={d:.3e} infidelity={f:.3e}"


def run_engine(module, mode, init=None, seed=1, physical=False):
    if init is not None:
        e = q.CUDAEngine(initial_state=init, seed=seed, mode=mode)
    else:
        e = q.CUDAEngine(module.num_qubits, seed=seed, mode=mode)
    if physical:
        e.set_option(1, 1)
    e.execute(module)
    return e


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_reference_fixtures(case, mode):
    e = run_engine(case.module, mode, init=case.init, seed=case.seed)
    check_close(case.expected, e.state())
    assert e.measurements() == case.meas


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n", [13, 14, 15, 17])
def test_zoo_all_types_vs_oracle(n, mode):
    m = zoo.random_circuit(n, 300, seed=n, types=zoo.REF_TYPES + zoo.EXT_TYPES, max_dense=6)
    ref, _ = oracle.run_oracle(m)
    check_close(ref, run_engine(m, mode).state())


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("types", [["h", "x", "cx", "ccx"], ["rz", "cz", "cp", "z", "s", "diag1", "diag2"],
                                   ["swap", "cswap", "u2", "x"], ["u3", "u4", "u5", "h"], ["u6", "rx", "cz"]])
def test_zoo_families_vs_oracle(types, mode):
    m = zoo.random_circuit(16, 200, seed=len(types) * 7, types=types, max_dense=6)
    ref, _ = oracle.run_oracle(m)
    check_close(ref, run_engine(m, mode).state())


@pytest.mark.parametrize("mode", MODES)
def test_random_h_rx_cx_20q_vs_reference(mode):
    """The 20-qubit, 40-layer H/RX/CX recipe, amplitude by amplitude."""
    m = circuits.random_h_rx_cx(20, 40, seed=2024)
    if oracle.reference_available():
        ref, _ = oracle.run_reference(m, seed=1)
    else:
        ref, _ = oracle.run_oracle(m)
    check_close(ref, run_engine(m, mode).state())


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("physical", [False, True])
def test_windowed_stream_executes_global_swap(mode, physical):
    case = next(c for c in CASES if c.name == "win_zoo10")
    check_close(case.expected, run_engine(case.module, mode, physical=physical).state())
    # a 16-qubit windowed stream with many swaps, built by the reference middle end
    if oracle.reference_available():
        m = zoo.random_circuit(16, 200, seed=99, types=["h", "rx", "cx", "swap", "ccx", "y", "s"])
        truth, _ = oracle.run_oracle(m)
        prog, data, meta = oracle.transpile_reference(m, fusion=False, hw=True, cost_model=1, k_safe=4)
        win = zoo.module_from_arrays(16, prog, data, meta)
        assert np.any(prog["type"] == GateType.GLOBAL_SWAP)
        check_close(truth, run_engine(win, mode, physical=physical).state())


@pytest.mark.parametrize("mode", MODES)
def test_random_rot_cz_and_qft(mode):
    m = circuits.random_rot_cz(18, 6, seed=3)
    ref, _ = oracle.run_oracle(m)
    check_close(ref, run_engine(m, mode).state())
    x = 0b1011001110101
    got = run_engine(circuits.qft(16, basis_state=x), mode).state()
    check_close(circuits.qft_expected(16, x), got, tol=1e-5, infid=1e-6)


def test_plain_and_tiled_agree_at_24_qubits():
    m = zoo.random_circuit(24, 400, seed=24, types=zoo.REF_TYPES + zoo.EXT_TYPES, max_dense=5)
    a = run_engine(m, "plain").state()
    b = run_engine(m, "tiled").state()
    c = run_engine(m, "tiled_tc").state()
    check_close(a, b)
    check_close(a, c)


@pytest.mark.parametrize("qubits", [[5, 6, 7, 8, 9], [9, 2, 12, 7, 0], [13, 1, 4, 10, 6]])
def test_tensor_core_dense5_vs_oracle(qubits):
    """One random 5-qubit unitary (a tensor-core op) on a random 14-qubit state."""
    rng = np.random.default_rng(sum(qubits))
    qc = QuantumCircuit(14)
    qc.unitary(qubits, zoo.random_unitary(5, rng))
    m = qc.release()
    init = zoo.random_state(14, 3)
    ref, _ = oracle.run_oracle(m, init=init)
    e = q.CUDAEngine(initial_state=init, mode="tiled_tc")
    e.execute(m)
    assert e.last_stats()["tc_ops"] >= 1
    check_close(ref, e.state())


def test_tensor_core_phase_fusion_vs_oracle():
    """Many gates on a few qubits: the planner fuses each register phase into
    tensor-core unitaries; thread-dependent CZs split them."""
    m = circuits.random_rot_cz(16, 10, seed=4)
    ref, _ = oracle.run_oracle(m)
    e = q.CUDAEngine(16, mode="tiled_tc")
    e.execute(m)
    assert e.last_stats()["tc_ops"] >= 1
    check_close(ref, e.state())
    m2 = zoo.random_circuit(15, 400, seed=77, types=["h", "rx", "ry", "rz", "cz", "cx", "u2", "s", "y"])
    ref2, _ = oracle.run_oracle(m2)
    check_close(ref2, run_engine(m2, "tiled_tc").state())


def test_measurement_seed_determinism_and_reset():
    """test_engine_measure.cpp:46-100."""
    qc = QuantumCircuit(1)
    qc.h(0).measure(0)
    m = qc.release()
    e = q.CUDAEngine(1, seed=42)
    e.execute(m)
    first = e.measurements()
    st = e.state()
    assert len(first) == 1
    assert abs(abs(st[first[0]]) ** 2 - 1.0) < 1e-6
    e.reset()
    assert e.measurements() == []
    assert abs(e.state()[0] - 1) < 1e-12
    e.set_seed(42)
    e.execute(m)
    assert e.measurements() == first
    ref, meas = oracle.run_oracle(m, seed=42)
    assert meas == first


def test_bell_shots_correlated():
    qc = QuantumCircuit(2)
    qc.h(0).cx(0, 1).measure([0, 1])
    m = qc.release()
    e = q.CUDAEngine(2, seed=5)
    for _ in range(100):
        e.reset()
        e.execute(m)
        ms = e.measurements()
        assert len(ms) == 2 and ms[0] == ms[1]


def test_measure_inside_tiled_program_matches_oracle():
    m = zoo.random_circuit(15, 120, seed=3, types=["h", "rx", "cx", "cz"])
    qc = QuantumCircuit(15)
    qc.measure([3, 7, 14])
    for g in qc.program():
        m.append(g)
    m2 = zoo.random_circuit(15, 60, seed=4, types=["h", "ry", "cx"])
    for g in m2.program():
        m.append(g)
    for mode in MODES:
        ref, meas = oracle.run_oracle(m, seed=11)
        e = run_engine(m, mode, seed=11)
        assert e.measurements() == meas
        check_close(ref, e.state())


def test_multi_block_handoff_stays_on_device():
    """CircuitRunner-style continuity (test_circuit_runner.cpp:229-307)."""
    b1 = circuits.random_h_rx_cx(14, 3, seed=1)
    b2 = circuits.random_rot_cz(14, 3, seed=2)
    e1 = q.CUDAEngine(14, seed=1)
    e1.execute(b1)
    sv = e1.extract_state_vector()
    assert not sv.empty() and sv.num_qubits() == 14
    e2 = q.CUDAEngine(state_vector=sv)
    assert sv.empty()
    e2.execute(b2)
    joined = IRModule(14)
    for g in list(b1.program()) + list(b2.program()):
        joined.append(g)
    ref, _ = oracle.run_oracle(joined)
    check_close(ref, e2.state())
    e3 = q.CUDAEngine(14)
    e3.set_state_vector(e2.extract_state_vector())
    check_close(ref, e3.state())


def test_initial_state_and_errors():
    init = zoo.random_state(10, 1)
    m = zoo.random_circuit(10, 50, seed=2)
    ref, _ = oracle.run_oracle(m, init=init)
    e = q.CUDAEngine(initial_state=init)
    e.execute(m)
    check_close(ref, e.state())
    e.reset(init)
    check_close(init, e.state())
    with pytest.raises(ValueError):
        q.CUDAEngine(initial_state=np.ones(3) / math.sqrt(3))        # not a power of 2
    with pytest.raises(ValueError):
        q.CUDAEngine(initial_state=np.ones(4))                        # not normalized
    bad = np.zeros(1, dtype=q._lib.GATE_INSTR_DTYPE)
    bad[0]["type"] = 0x7F
    with pytest.raises(RuntimeError):
        e.execute(bad)
    with pytest.raises(ValueError):
        e.execute(np.array([make_instr(GateType.H, [10])]))
    with pytest.raises(ValueError):
        e.execute(np.array([make_instr(GateType.UNITARY, [0], matrix_idx=3)]))


def test_state_vector_api():
    """test_state_vector.cpp:14-47."""
    sv = q.CUDAStateVector()
    assert sv.empty()
    sv.initialize(3)
    assert sv.num_qubits() == 3 and sv.dimension() == 8 and not sv.empty()
    a = sv.amplitudes()
    assert a[0] == 1 and np.all(a[1:] == 0)
    sv.initialize(zoo.random_state(4, 3))
    assert sv.num_qubits() == 4


def test_fp64_reductions():
    m = zoo.random_circuit(18, 200, seed=18, types=["h", "rx", "ry", "cx", "cz"])
    ref, _ = oracle.run_oracle(m)
    e = run_engine(m, "tiled")
    st = e.state()
    p = np.abs(st) ** 2
    assert abs(e.norm_sq() - p.sum()) < 1e-12
    idx = np.arange(p.size)
    for qb in (0, 5, 12, 17):
        assert abs(e.prob_one(qb) - p[(idx >> qb) & 1 == 1].sum()) < 1e-12
    ez = e.expect_z()
    want = np.array([p.sum() - 2 * p[(idx >> qb) & 1 == 1].sum() for qb in range(18)])
    assert np.max(np.abs(ez - want)) < 1e-10
    pr = np.abs(ref) ** 2
    want_ref = np.array([1 - 2 * pr[(idx >> qb) & 1 == 1].sum() for qb in range(18)])
    assert np.max(np.abs(ez - want_ref)) < 1e-5


@pytest.mark.parametrize("n", [3, 12, 16])
def test_sampling_distribution_and_determinism(n):
    m = zoo.random_circuit(n, 20 * n, seed=n, types=["h", "ry", "cx"])
    e = run_engine(m, "plain")
    st = e.state()
    p = np.abs(st) ** 2
    shots = 200000
    s1 = e.sample(1234, shots)
    s2 = e.sample(1234, shots)
    assert np.array_equal(s1, s2)
    assert np.all(s1 < p.size) and np.all(p[s1.astype(np.int64)] > 0)
    counts = np.bincount(s1.astype(np.int64), minlength=p.size) / shots
    tvd = 0.5 * np.abs(counts - p).sum()
    assert tvd < 0.02 + 3 * math.sqrt(p.size / shots)

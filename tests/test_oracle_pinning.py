"""The oracle (oracle/sv_oracle.c) pinned against the reference: its own
known-answer tests, fixtures generated by the unmodified reference engine,
and (where oracle/_ref is built) live runs of the reference."""
import math

import numpy as np
import pytest

from golden_cases import load_cases
from oracle import oracle
from qlassical_b200 import circuits
from qlassical_b200.ir import GateType, QuantumCircuit, make_instr
import zoo

CASES = load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_oracle_matches_reference_fixture(case):
    st, meas = oracle.run_oracle(case.module, init=case.init, seed=case.seed)
    assert oracle.max_abs_diff(st, case.expected) < 1e-12
    assert meas == case.meas


def test_oracle_reproduces_reference_global_swap_noop():
    """With GLOBAL_SWAP as a no-op (cpu_openmp_engine.hpp:217-219) the
    windowed stream gives the reference's wrong answer."""
    case = next(c for c in CASES if c.name == "win_zoo10")
    good, _ = oracle.run_oracle(case.module, seed=1)
    bad, _ = oracle.run_oracle(case.module, seed=1, global_swap_noop=True)
    assert oracle.max_abs_diff(good, case.expected) < 1e-12
    assert oracle.max_abs_diff(bad, case.expected) > 1e-3


def _state(prog_gates, n, init=None, seed=0):
    from qlassical_b200.ir import IRModule
    m = IRModule(n)
    for g in prog_gates:
        m.append(g)
    return oracle.run_oracle(m, init=init, seed=seed)


T = GateType
R2 = 1 / math.sqrt(2)


def test_kat_single_qubit():
    """test_engine_kernels.cpp:48-116."""
    s, _ = _state([make_instr(T.X, [0])], 1)
    assert abs(s[1] - 1) < 1e-6 and abs(s[0]) < 1e-6
    s, _ = _state([make_instr(T.H, [0])], 1)
    assert abs(s[0].real - R2) < 1e-6 and abs(s[1].real - R2) < 1e-6
    s, _ = _state([make_instr(T.Y, [0])], 1)
    assert abs(s[1].imag - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.Z, [0])], 1)
    assert abs(s[1].real + 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.S, [0])], 1)
    assert abs(s[1].imag - 1) < 1e-6
    s, _ = _state([make_instr(T.RX, [0], param=math.pi)], 1)
    assert abs(s[1].imag + 1) < 1e-6
    s, _ = _state([make_instr(T.RY, [0], param=math.pi / 2)], 1)
    assert abs(s[0].real - R2) < 1e-6 and abs(s[1].real - R2) < 1e-6


def test_kat_routing():
    """test_engine_kernels.cpp:118-171 (index convention: qubit q = bit q)."""
    s, _ = _state([make_instr(T.X, [2]), make_instr(T.CX, [2, 0])], 3)
    assert abs(s[5] - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.CX, [0, 2])], 3)
    assert abs(s[5] - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.SWAP, [0, 2])], 3)
    assert abs(s[4] - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [2]), make_instr(T.SWAP, [2, 0])], 3)
    assert abs(s[1] - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.X, [1]), make_instr(T.CCX, [1, 0, 2])], 3)
    assert abs(s[7] - 1) < 1e-6
    s, _ = _state([make_instr(T.X, [0]), make_instr(T.X, [1]), make_instr(T.CSWAP, [1, 0, 2])], 3)
    assert abs(s[6] - 1) < 1e-6


def test_kat_unitary_convention():
    """test_engine_kernels.cpp:173-202: matrix bit i <-> instr.qubits[i]."""
    qc = QuantumCircuit(3)
    sw = np.zeros((4, 4), dtype=complex)
    sw[0, 0] = sw[1, 2] = sw[2, 1] = sw[3, 3] = 1
    qc.x(0).unitary([0, 2], sw)
    s, _ = oracle.run_oracle(qc.release())
    assert abs(s[1]) < 1e-6 and abs(s[4] - 1) < 1e-6


def test_kat_kickback_and_bell_measure():
    """test_engine_kernels.cpp:204-230, test_engine_measure.cpp:103-124."""
    s, _ = _state([make_instr(T.H, [0]), make_instr(T.X, [1]), make_instr(T.H, [1]), make_instr(T.CX, [0, 1])], 2)
    assert np.allclose(s.real, [0.5, -0.5, -0.5, 0.5], atol=1e-6)
    for seed in range(100):
        _, ms = _state([make_instr(T.H, [0]), make_instr(T.CX, [0, 1]), make_instr(T.MEASURE, [0]),
                        make_instr(T.MEASURE, [1])], 2, seed=seed)
        assert len(ms) == 2 and ms[0] == ms[1]


def test_rng_matches_std_mt19937_64():
    """MT19937-64 restatement: the 10000th output of std::mt19937_64 with
    the default seed 5489 is 9981545732273789042 (C++ [rand.predef])."""
    import ctypes
    L = ctypes.CDLL(oracle.ORACLE_SO)
    L.orc_rng_create.restype = ctypes.c_void_p
    L.orc_rng_create.argtypes = [ctypes.c_uint64]
    L.orc_rng_next.restype = ctypes.c_uint64
    L.orc_rng_next.argtypes = [ctypes.c_void_p]
    L.orc_rng_destroy.argtypes = [ctypes.c_void_p]
    g = L.orc_rng_create(5489)
    for _ in range(9999):
        L.orc_rng_next(g)
    v = L.orc_rng_next(g)
    L.orc_rng_destroy(g)
    assert v == 9981545732273789042


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_live_reference(seed):
    n = 6 + seed
    m = zoo.random_circuit(n, 150, seed=1000 + seed)
    a, _ = oracle.run_oracle(m, seed=3)
    b, _ = oracle.run_reference(m, seed=3)
    assert oracle.max_abs_diff(a, b) < 1e-12


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_oracle_matches_reference_on_cz_cp_as_unitary():
    """The additive CZ / CP types agree with the reference executing them as
    2-qubit UNITARY diagonals."""
    m = circuits.random_rot_cz(10, 6, seed=5)
    ref, _ = oracle.run_reference(circuits.to_reference_ir(m), seed=1)
    orc, _ = oracle.run_oracle(m, seed=1)
    assert oracle.max_abs_diff(ref, orc) < 1e-12


def test_qft_circuit_matches_analytic_dft():
    """The QFT generator computes exp(2 pi i x k / 2^n); the residual comes
    from the CP angles being stored as float32 in the IR (frontend.hpp:93),
    so the tolerance is 1e-6 rather than FP64 round-off."""
    for n in (3, 5, 8):
        for x in (0, 1, (1 << n) - 3):
            s, _ = oracle.run_oracle(circuits.qft(n, basis_state=x))
            assert oracle.max_abs_diff(s, circuits.qft_expected(n, x)) < 1e-6


@pytest.mark.parametrize("n,depth,seed", [(7, 3, 1), (12, 5, 1234), (30, 24, 1234)])
def test_ref_workloads_match_package_circuits(n, depth, seed):
    """bench.py's reference arm builds the benchmark circuit with numpy alone
    (oracle/ref_workloads.py); its records and pool are byte-identical to the
    package's circuit rewritten into the reference IR."""
    from oracle import ref_workloads
    rc = ref_workloads.random_rot_cz(n, depth, seed=seed)
    m = circuits.to_reference_ir(circuits.random_rot_cz(n, depth, seed=seed))
    assert rc.prog.tobytes() == m.program().tobytes()
    pool = m.unitaries()
    assert np.array_equal(rc.pool_data, pool.data)
    assert rc.pool_meta.tobytes() == pool.metadata().tobytes()
    assert rc.layer_starts == [i * (n + n // 2) for i in range(depth)]
    one = rc.layers(2, 1)
    assert one.gate_count() == n + n // 2
    assert one.prog.tobytes() == m.program()[2 * (n + n // 2):3 * (n + n // 2)].tobytes()


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_ref_workloads_run_through_reference():
    """The numpy-built reference IR runs through the reference engine (and
    its transpiler) and agrees with the oracle on the package's circuit."""
    from oracle import ref_workloads
    rc = ref_workloads.random_rot_cz(9, 4, seed=3)
    a, _ = oracle.run_reference(rc, seed=1)
    b, _ = oracle.run_oracle(circuits.random_rot_cz(9, 4, seed=3))
    assert oracle.max_abs_diff(a, b) < 1e-12
    prog, data, meta = oracle.transpile_reference(rc, fusion=True, hw=False)
    fused = ref_workloads.RefCircuit(9, prog, data, meta)
    c, _ = oracle.run_reference(fused, seed=1)
    assert oracle.max_abs_diff(a, c) < 1e-10
    assert oracle.time_reference(fused, reps=1) > 0.0


@pytest.mark.parametrize("n", [3, 8, 33])
def test_ref_workloads_qft_matches_package(n):
    from oracle import ref_workloads
    rc = ref_workloads.qft(n)
    m = circuits.to_reference_ir(circuits.qft(n))
    assert rc.prog.tobytes() == m.program().tobytes()
    assert np.array_equal(rc.pool_data, m.unitaries().data)
    assert rc.pool_meta.tobytes() == m.unitaries().metadata().tobytes()

"""The FP64 checker (a complex128 device state run gate by gate in double
precision) against the oracle: it is the yardstick for the complex64
engine at sizes the host oracle cannot reach quickly, so it must agree with
the oracle to FP64 rounding (1e-12) on every instruction type it accepts."""
import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import circuits
from oracle import oracle
import zoo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [10, 14, 17])
def test_check64_zoo_vs_oracle(n):
    m = zoo.random_circuit(n, 250, seed=100 + n, types=zoo.REF_TYPES + zoo.EXT_TYPES, max_dense=6)
    ref, _ = oracle.run_oracle(m)
    c = q.Check64(n)
    c.execute(m)
    got = c.state()
    assert oracle.max_abs_diff(ref, got) < 1e-12
    assert abs(oracle.infidelity(ref, got)) < 1e-12


def test_check64_windowed_stream_vs_oracle():
    """GLOBAL_SWAPs of a windowed, fused stream permute physical qubits; the
    result is the logical state of the unfused circuit."""
    from qlassical_b200.middleware import Middleware, TranspilerConfig
    m = circuits.random_rot_cz(16, 8, seed=5)
    w = Middleware().transpile(m, config=TranspilerConfig(max_fusion_qubits=5, k_safe=9))
    assert np.any(w.program()["type"] == q.GateType.GLOBAL_SWAP)
    ref, _ = oracle.run_oracle(m)
    c = q.Check64(16)
    c.execute(w)
    assert oracle.max_abs_diff(ref, c.state()) < 1e-12


def test_check64_compare_matches_host_formula():
    """qlb_check64_compare reduces max|delta| and the infidelity over the
    whole state exactly as the host formula does on the downloaded states."""
    m = circuits.random_rot_cz(15, 6, seed=9)
    c = q.Check64(15)
    c.execute(m)
    e = q.CUDAEngine(15, mode="tiled")
    e.execute(m)
    r = c.compare(e)
    ref, got = c.state(), e.state()
    assert abs(r["max_abs_diff"] - oracle.max_abs_diff(ref, got)) < 1e-15
    assert abs(r["infidelity"] - oracle.infidelity(ref, got)) < 1e-12
    assert abs(r["norm_ref"] - 1.0) < 1e-12
    assert r["max_abs_diff"] < 2e-6 and r["infidelity"] < 1e-9


def test_check64_rejects_measure():
    qc = q.QuantumCircuit(4)
    qc.h(0)
    qc.measure(0)
    c = q.Check64(4)
    with pytest.raises(ValueError):          # QLB_ERR_INVALID_ARG
        c.execute(qc.release())

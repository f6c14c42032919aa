"""Parity of the benchmarked pipeline: the random RX/RY/RZ + CZ-pairs circuit
of depth 24, transpiled by the GPU middle end exactly as the benchmark does
(fusion into dense blocks of up to 5 qubits, qubit windowing with k_safe =
the tile window, reference middleware.hpp:466-524, 759-860), executed on the
tensor-core tile path and on the FP32 tile path, and compared with the FP64
result of the *unfused* circuit: the oracle (complex128, host) at 20 and 24
qubits, the FP64 checker (complex128, device) at 26 qubits.  Tolerances as
everywhere: max |delta amplitude| <= 2e-5, infidelity <= 1e-6."""
import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import circuits
from qlassical_b200.middleware import Middleware, TranspilerConfig, gpu_safe_qubit_limit
from oracle import oracle

pytestmark = pytest.mark.gpu

MAX_DIFF = 2e-5
MAX_INFID = 1e-6


def headline_stream(n, depth=24, seed=1234):
    m = circuits.random_rot_cz(n, depth, seed=seed)
    cfg = TranspilerConfig(max_fusion_qubits=5, k_safe=gpu_safe_qubit_limit())
    fused = Middleware().transpile(m, config=cfg)
    prog = fused.program()
    # the stream is the benchmarked form: 5-qubit dense blocks and window swaps
    assert np.any(prog["type"] == q.GateType.GLOBAL_SWAP)
    assert np.any((prog["type"] == q.GateType.FUSED_BLOCK) & ((prog["flags_arity"] & 0x0F) == 5))
    return m, fused


@pytest.mark.parametrize("n", [20, 24])
def test_headline_pipeline_vs_oracle(n):
    m, fused = headline_stream(n)
    ref, _ = oracle.run_oracle(m)
    for mode in ("tiled_tc", "tiled"):
        e = q.CUDAEngine(n, mode=mode)
        e.execute(fused)
        if mode == "tiled_tc":
            assert e.last_stats()["tc_ops"] >= 1
        got = e.state()
        d = oracle.max_abs_diff(ref, got)
        f = oracle.infidelity(ref, got)
        assert d <= MAX_DIFF and f <= MAX_INFID, (mode, d, f)


def test_headline_pipeline_26q_vs_fp64_checker():
    n = 26
    m, fused = headline_stream(n)
    c = q.Check64(n)
    c.execute(m)
    for mode in ("tiled_tc", "tiled"):
        e = q.CUDAEngine(n, mode=mode)
        e.execute(fused)
        r = c.compare(e)
        assert r["max_abs_diff"] <= MAX_DIFF and r["infidelity"] <= MAX_INFID, (mode, r)
        del e

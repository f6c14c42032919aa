"""The tensor-core chain kernel (chain.cu) against the oracle and against
the general tile kernel on the same plans (QLB_OPT_TC_CHAIN off): chain
passes of both load paths (cp.async pieces for short runs, bulk copies for
runs >= 4 KB), a phase-0 op written in its own rows and entry-scattered
first ops, grids smaller than the SM count, and passes of one to several
tensor-core ops."""
import numpy as np
import pytest

import qlassical_b200 as q
from qlassical_b200 import circuits
from qlassical_b200.middleware import Middleware, TranspilerConfig
from oracle import oracle
import zoo

pytestmark = pytest.mark.gpu

MAX_DIFF = 2e-5
MAX_INFID = 1e-6
QLB_OPT_TC_CHAIN = 3


def run(module, chain, init=None):
    e = q.CUDAEngine(module.num_qubits, mode="tiled_tc") if init is None else \
        q.CUDAEngine(initial_state=init, mode="tiled_tc")
    e.set_option(QLB_OPT_TC_CHAIN, 1 if chain else 0)
    e.execute(module)
    return e.state(), e.last_stats()


def check(ref, got):
    d, f = oracle.max_abs_diff(ref, got), oracle.infidelity(ref, got)
    assert d <= MAX_DIFF and f <= MAX_INFID, (d, f)


@pytest.mark.parametrize("n", [14, 18, 22])
def test_chain_on_the_fused_rotation_circuit(n):
    m = circuits.random_rot_cz(n, 16, seed=n)
    f = Middleware().transpile(m, config=TranspilerConfig(max_fusion_qubits=5))
    ref, _ = oracle.run_oracle(m)
    on, st_on = run(f, True)
    off, st_off = run(f, False)
    assert st_on["chain_passes"] >= 1 and st_off["chain_passes"] == 0
    check(ref, on)
    check(ref, off)
    assert oracle.max_abs_diff(on, off) < 2e-6


@pytest.mark.parametrize("low", [True, False])
def test_chain_dense5_blocks_bulk_and_short_runs(low):
    """5-qubit unitaries on qubits 0..12 of a 16-qubit state: the tile is
    qubits 0..12 (one 64 KB run: bulk copies); on scattered qubits the
    tiles have short runs (cp.async pieces)."""
    n = 16
    rng = np.random.default_rng(7 if low else 8)
    qc = q.QuantumCircuit(n)
    pool = list(range(13)) if low else list(range(n))
    for _ in range(6):
        qs = [int(x) for x in rng.permutation(pool)[:5]]
        qc.unitary(qs, zoo.random_unitary(5, rng))
    m = qc.release()
    init = zoo.random_state(n, 5)
    ref, _ = oracle.run_oracle(m, init=init)
    got, st = run(m, True, init=init)
    assert st["chain_passes"] >= 1, st
    check(ref, got)


def test_chain_single_op_passes_and_small_grid():
    """One 5-qubit unitary on a 13-qubit state (one tile, one CTA) and on a
    14-qubit state (two tiles)."""
    for n in (13, 14):
        rng = np.random.default_rng(n)
        qc = q.QuantumCircuit(n)
        qc.unitary([int(x) for x in rng.permutation(n)[:5]], zoo.random_unitary(5, rng))
        m = qc.release()
        init = zoo.random_state(n, 9)
        ref, _ = oracle.run_oracle(m, init=init)
        got, st = run(m, True, init=init)
        assert st["chain_passes"] >= 1 and st["tc_ops"] >= 1, st
        check(ref, got)


@pytest.mark.parametrize("n", [15, 17])
@pytest.mark.parametrize("signs_only", [True, False])
def test_chain_post_terms_of_the_last_pass(n, signs_only):
    """CZs that end the circuit (across out-of-tile and in-tile qubits) are
    applied by the chain kernel's producers as sign flips while the last
    pass stores each tile; with an RZ and a CP among them they stay a
    diagonal op of the general kernel."""
    from test_planner_emulated import _ends_with_diagonals
    from qlassical_b200.engine import describe_plan
    m = _ends_with_diagonals(n, n, signs_only)
    plan = describe_plan(m, n, "tiled_tc")
    assert (plan["passes"][-1]["post_n"] >= 2) == signs_only
    init = zoo.random_state(n, 4)
    ref, _ = oracle.run_oracle(m, init=init)
    on, _ = run(m, True, init=init)
    off, _ = run(m, False, init=init)
    check(ref, on)
    check(ref, off)

"""Batched mode (qlb_batch_*): many circuits per launch, one CUDA graph per
run.  Per-circuit results equal execute() + expect_z() on |0...0>: checked
against the FP64 oracle (small sizes) and against the single-circuit
engine; a circuit's results do not depend on the rest of its batch."""
import numpy as np
import pytest

from oracle import oracle
import qlassical_b200 as q
from qlassical_b200 import circuits
from qlassical_b200.batch import Batch, run_batch
from qlassical_b200.ir import QuantumCircuit


def test_hea_batch_distribution():
    mods = circuits.hea_batch(512, seed=3)
    ns = np.array([m.num_qubits for m in mods])
    assert ns.min() >= 10 and ns.max() <= 20
    # log-uniform: about half of the circuits below sqrt(10*20) ~ 14.1 qubits
    assert 0.35 < np.mean(ns <= 14) < 0.65
    gates = np.array([m.gate_count() for m in mods])
    # per layer 2n rotations + (n-1) CZ, depth 8..32
    assert np.all(gates >= 8 * (3 * ns - 1)) and np.all(gates <= 32 * (3 * ns - 1))


def test_expect_z_helper_matches_definition():
    st = np.zeros(8, dtype=np.complex128)
    st[5] = 1.0                   # |101>: q0 = 1, q1 = 0, q2 = 1
    assert np.allclose(circuits.expect_z_of(st, 3), [-1.0, 1.0, -1.0])


def _oracle_ez(m):
    st, _ = oracle.run_oracle(m)
    return circuits.expect_z_of(st, m.num_qubits), st


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled", "tiled_tc", "auto"])
def test_batch_matches_oracle(mode):
    mods = circuits.hea_batch(24, seed=11, n_min=10, n_max=15, d_min=4, d_max=10)
    b = Batch(mods, mode)
    b.run()
    b.synchronize()
    ez = b.expect_z()
    for i, m in enumerate(mods):
        want, st = _oracle_ez(m)
        assert np.max(np.abs(ez[i] - want)) < 2e-5, (i, m.num_qubits)
        if i < 4:
            got = b.state(i)
            assert oracle.infidelity(st, got) < 1e-6


@pytest.mark.gpu
def test_batch_matches_single_engine_on_mixed_sizes():
    mods = circuits.hea_batch(64, seed=5, n_min=10, n_max=20, d_min=8, d_max=16)
    ez = run_batch(mods, "tiled")
    for i in range(0, 64, 7):
        m = mods[i]
        eng = q.CUDAEngine(m.num_qubits, mode="tiled")
        eng.execute(m)
        assert np.max(np.abs(ez[i] - eng.expect_z())) < 1e-5, i


@pytest.mark.gpu
def test_alone_vs_mix_bitwise_identical():
    mods = circuits.hea_batch(16, seed=8, n_min=12, n_max=18, d_min=6, d_max=12)
    mixed = Batch(mods, "tiled")
    mixed.run()
    mixed.synchronize()
    ez_mix = mixed.expect_z()
    for i in (0, 5, 11):
        alone = Batch([mods[i]], "tiled")
        alone.run()
        alone.synchronize()
        assert np.array_equal(alone.expect_z()[0], ez_mix[i])
        assert np.array_equal(alone.state(0), mixed.state(i))


@pytest.mark.gpu
def test_batch_rerun_is_deterministic_and_resets():
    mods = circuits.hea_batch(8, seed=21, n_min=11, n_max=16, d_min=5, d_max=8)
    b = Batch(mods, "tiled")
    b.run()
    b.synchronize()
    first = b.expect_z()
    b.run()
    b.run()
    b.synchronize()
    for x, y in zip(first, b.expect_z()):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_batch_edge_cases():
    empty = QuantumCircuit(5).release()            # no gates: |00000>
    x1 = QuantumCircuit(1)
    x1.x(0)
    ez = run_batch([empty, x1.release()], "tiled")
    assert np.allclose(ez[0], np.ones(5)) and np.allclose(ez[1], [-1.0])
    qc = QuantumCircuit(3)
    qc.h(0)
    qc.measure(0)
    with pytest.raises(ValueError):
        Batch([qc.release()], "tiled")
    with pytest.raises(ValueError):
        Batch([], "tiled")


@pytest.mark.gpu
def test_autotuner_search_is_recorded_and_results_hold():
    """mode "auto": one tune entry per size class, every candidate timed on
    its sample, one mode for the batch and per class the fastest fixed-low
    count in it, and every circuit's <Z> still matches the oracle whichever
    configuration planned it."""
    mods = circuits.hea_batch(40, seed=13, n_min=10, n_max=17, d_min=4, d_max=10)
    b = Batch(mods, "auto")
    b.run()
    b.synchronize()
    st = b.stats()
    sizes = sorted({max(13, m.num_qubits) for m in mods})
    assert [t["num_qubits"] for t in st["tune"]] == sizes
    assert sum(t["circuits"] for t in st["tune"]) == len(mods)
    assert len({t["best"]["mode"] for t in st["tune"]}) == 1
    for t in st["tune"]:
        assert 1 <= t["sample"] <= t["circuits"]
        assert all(x > 0 for x in t["ms"]), t
        base = 0 if t["best"]["mode"] == "tiled" else 3
        best = min(range(base, base + 3), key=lambda k: t["ms"][k])
        assert t["best"] == q._lib.batch_tune_candidate(best)
    assert st["tune_seconds"] > 0 and st["autotune_ms"][0] <= st["autotune_ms"][1] + 1e-9
    ez = b.expect_z()
    for i, m in enumerate(mods):
        want, _ = _oracle_ez(m)
        assert np.max(np.abs(ez[i] - want)) < 5e-5, (i, m.num_qubits)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
@pytest.mark.parametrize("tile_low", [4, 5, 6])
def test_engine_tile_low_option(mode, tile_low):
    """QLB_OPT_TILE_LOW on the single-circuit engine: same state as the oracle."""
    m = circuits.hea(17, 10, 3)
    e = q.CUDAEngine(17, mode=mode)
    e.set_option(q._lib.OPT_TILE_LOW, tile_low)
    e.execute(m)
    st, _ = oracle.run_oracle(m)
    assert oracle.max_abs_diff(st, e.state()) < 2e-5
    with pytest.raises(ValueError):
        e.set_option(q._lib.OPT_TILE_LOW, 7)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled_tc", "auto"])
def test_batch_fused_circuits_match_oracle(mode):
    """fuse=5: each circuit is fused by the GPU middle end (blocks of up to 5
    qubits) before planning; <Z> still match the oracle."""
    mods = circuits.hea_batch(24, seed=17, n_min=10, n_max=16, d_min=4, d_max=10)
    b = Batch(mods, mode, fuse=5)
    b.run()
    b.synchronize()
    ez = b.expect_z()
    for i, m in enumerate(mods):
        want, _ = _oracle_ez(m)
        assert np.max(np.abs(ez[i] - want)) < 5e-5, (i, m.num_qubits)
    assert b.stats()["amp_updates"] == sum(m.gate_count() * 2 ** m.num_qubits for m in mods)
    with pytest.raises(ValueError):
        Batch(mods[:2], "tiled_tc", fuse=6)

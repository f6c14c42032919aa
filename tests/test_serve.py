"""Serving loop (qlb_server_*): continuous batching of circuit requests.
Results are checked against the FP64 oracle (<Z>), statistically for
samples, and bitwise between a request served alone and the same request
served among others."""
import numpy as np
import pytest

from oracle import oracle
from qlassical_b200 import circuits
from qlassical_b200.ir import QuantumCircuit


def test_serving_workload_distribution():
    mods = circuits.serving_requests(400, seed=3)
    ns = np.array([m.num_qubits for m in mods])
    assert ns.min() >= 12 and ns.max() <= 30
    assert 0.35 < np.mean(ns <= 19) < 0.65          # log-uniform median ~ sqrt(12*30) ~ 19
    t = circuits.poisson_arrivals(2000, rate_hz=50.0, seed=1)
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 0.02) < 0.002 and np.all(gaps > 0)


@pytest.mark.gpu
def test_serve_matches_oracle_and_samples():
    from qlassical_b200.serve import Server
    mods = circuits.serving_requests(12, seed=5, n_min=12, n_max=15, d_min=4, d_max=8)
    with Server(memory_bytes=1 << 30) as srv:
        ids = [srv.submit(m, shots=4096, seed=100 + i) for i, m in enumerate(mods)]
        res = [srv.result(i) for i in ids]
    for m, r in zip(mods, res):
        st, _ = oracle.run_oracle(m)
        want = circuits.expect_z_of(st, m.num_qubits)
        assert np.max(np.abs(r.expect_z - want)) < 2e-5
        assert r.samples.max() < (1 << m.num_qubits)
        # per-qubit marginals of the samples vs the oracle's P(q=1)
        p1 = (1.0 - want) / 2.0
        bits = ((r.samples[:, None] >> np.arange(m.num_qubits, dtype=np.uint64)) & np.uint64(1)).astype(float)
        assert np.max(np.abs(bits.mean(axis=0) - p1)) < 5.0 * 0.5 / np.sqrt(4096) + 1e-3
        assert r.t_submit <= r.t_admit <= r.t_done


@pytest.mark.gpu
def test_serve_alone_vs_mix_identical():
    from qlassical_b200.serve import Server
    mods = circuits.serving_requests(10, seed=9, n_min=12, n_max=18, d_min=6, d_max=12)
    target = mods[3]
    with Server(memory_bytes=1 << 30) as srv:
        alone = srv.result(srv.submit(target, shots=1024, seed=77))
    with Server(memory_bytes=1 << 30) as srv:
        ids = [srv.submit(m, shots=256, seed=i) for i, m in enumerate(mods[:3])]
        tid = srv.submit(target, shots=1024, seed=77)
        ids += [srv.submit(m, shots=256, seed=i) for i, m in enumerate(mods[4:])]
        mixed = srv.result(tid)
        for i in ids:
            srv.result(i)
    assert np.array_equal(alone.expect_z, mixed.expect_z)
    assert np.array_equal(alone.samples, mixed.samples)


@pytest.mark.gpu
def test_serve_admission_and_edge_cases():
    from qlassical_b200.serve import Server
    with Server(memory_bytes=2 << 20) as srv:     # 2 MiB arena: a 20-qubit state (8 MiB) cannot fit
        with pytest.raises(MemoryError):
            srv.submit(circuits.random_h_rx_cx(20, 2, seed=1), shots=16)
        empty = QuantumCircuit(3).release()
        r = srv.result(srv.submit(empty, shots=8, seed=1))
        assert np.allclose(r.expect_z, 1.0) and np.all(r.samples == 0)
        # more requests than fit at once (three 512 KiB states): admitted as blocks free up
        mods = [circuits.random_h_rx_cx(16, 3, seed=s) for s in range(12)]   # 512 KiB states
        ids = [srv.submit(m, shots=0, seed=0) for m in mods]
        for m, i in zip(mods, ids):
            got = srv.result(i).expect_z
            st, _ = oracle.run_oracle(m)
            assert np.max(np.abs(got - circuits.expect_z_of(st, 16))) < 2e-5
        qc = QuantumCircuit(2)
        qc.measure(0)
        with pytest.raises(ValueError):
            srv.submit(qc.release())


@pytest.mark.gpu
def test_serve_cancel_queued_and_admitted():
    """Host-side fault handling: cancelled requests leave the queue or the
    running rounds, release their device memory, and do not disturb the
    requests that share the server."""
    import time
    from qlassical_b200.serve import Server
    with Server(memory_bytes=2 << 20) as srv:       # room for one 17-qubit request (1 MiB state)
        a = circuits.random_h_rx_cx(17, 30, seed=1)
        b = circuits.random_h_rx_cx(17, 30, seed=2)
        ia = srv.submit(a, shots=0)
        ib = srv.submit(b, shots=0)                  # waits for a's memory
        srv.cancel(ib)
        with pytest.raises(RuntimeError):
            srv.result(ib)
        got = srv.result(ia).expect_z
        st, _ = oracle.run_oracle(a)
        assert np.max(np.abs(got - circuits.expect_z_of(st, 17))) < 2e-5
    with Server(memory_bytes=12 << 30) as srv:
        big = srv.submit(circuits.random_h_rx_cx(30, 40, seed=3), shots=0)   # ~1 s of rounds
        time.sleep(0.1)
        assert srv.stats()["active"] == 1
        srv.cancel(big)                              # admitted: leaves at the next round boundary
        with pytest.raises(RuntimeError):
            srv.result(big)
        deadline = time.time() + 5.0
        while srv.stats()["arena_used"] != 0 and time.time() < deadline:
            time.sleep(0.01)
        assert srv.stats()["arena_used"] == 0
        c = circuits.random_h_rx_cx(14, 5, seed=4)
        st, _ = oracle.run_oracle(c)
        assert np.max(np.abs(srv.result(srv.submit(c, shots=0)).expect_z - circuits.expect_z_of(st, 14))) < 2e-5


@pytest.mark.gpu
def test_serve_fuses_large_requests():
    """fuse_from: requests of at least that many qubits are fused by the GPU
    middle end (blocks of up to 5 qubits) and planned for the tensor cores;
    their <Z> still match the oracle, and the smaller requests are served
    exactly as without fusion (bitwise)."""
    from qlassical_b200.serve import Server
    mods = circuits.serving_requests(10, seed=6, n_min=12, n_max=17, d_min=6, d_max=12)
    assert any(m.num_qubits >= 15 for m in mods) and any(m.num_qubits < 15 for m in mods)
    with Server(memory_bytes=1 << 30, fuse_from=15) as srv:
        res = [srv.result(srv.submit(m, shots=256, seed=i)) for i, m in enumerate(mods)]
    with Server(memory_bytes=1 << 30) as srv:
        plain = [srv.result(srv.submit(m, shots=256, seed=i)) for i, m in enumerate(mods)]
    for m, r, p in zip(mods, res, plain):
        st, _ = oracle.run_oracle(m)
        assert np.max(np.abs(r.expect_z - circuits.expect_z_of(st, m.num_qubits))) < 2e-5
        if m.num_qubits < 15:
            assert np.array_equal(r.expect_z, p.expect_z) and np.array_equal(r.samples, p.samples)

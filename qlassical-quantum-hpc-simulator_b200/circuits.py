"""Seeded workload generators (synthetic; the reference ships no dataset).

Every generator draws from numpy's PCG64 generator seeded with `seed`, so a
(seed, sizes) pair names one circuit exactly.  Rotation angles are stored as
float32, as the reference builder does (frontend.hpp:280-292).

  random_h_rx_cx     20-qubit, 40-layer H/RX + nearest-neighbour CX circuit
  random_rot_cz      30-qubit depth-24 RX/RY/RZ + random disjoint CZ pairs
  qft                quantum Fourier transform: H + CP(pi/2^j) ladders + swaps
  hea                hardware-efficient ansatz layer (RY, RZ, CZ ladder)
  hea_batch          the batched workload: HEA circuits with log-uniform
                     sizes in [10, 20] qubits and depths U{8..32}
  serving_requests   the served workload: random_h_rx_cx circuits with
                     log-uniform sizes in [12, 30] qubits, depths U{10..40}
  poisson_arrivals   request arrival times of a Poisson process
  clustered          the reference benchmark's clustered H + CX-chain circuit
                     (benchmarks/bench_hw_awareness.cpp:30-53)
"""
from __future__ import annotations

import math

import numpy as np

from .ir import GateType, IRModule, QuantumCircuit, UnitaryPool, make_instr


def random_h_rx_cx(n: int = 20, layers: int = 40, seed: int = 1234) -> IRModule:
    """Per layer: H or RX(theta~U[0,2pi)) on every qubit (type drawn from the
    seeded stream), then CX(i, i+1) at even i in even layers, odd i in odd
    layers.  No fusion."""
    rng = np.random.default_rng(seed)
    qc = QuantumCircuit(n)
    for layer in range(layers):
        kinds = rng.integers(0, 2, size=n)
        thetas = rng.uniform(0.0, 2.0 * math.pi, size=n)
        for q in range(n):
            if kinds[q] == 0:
                qc.h(q)
            else:
                qc.rx(q, thetas[q])
        for i in range(layer % 2, n - 1, 2):
            qc.cx(i, i + 1)
    return qc.release()


def random_rot_cz(n: int = 30, depth: int = 24, seed: int = 1234) -> IRModule:
    """Per layer: RX/RY/RZ(theta~U[0,2pi)) on every qubit (type drawn from
    the seeded stream), then CZ on seeded random disjoint pairs covering the
    full qubit range."""
    rng = np.random.default_rng(seed)
    qc = QuantumCircuit(n)
    for _ in range(depth):
        kinds = rng.integers(0, 3, size=n)
        thetas = rng.uniform(0.0, 2.0 * math.pi, size=n)
        for q in range(n):
            (qc.rx, qc.ry, qc.rz)[kinds[q]](q, thetas[q])
        perm = rng.permutation(n)
        for i in range(0, n - 1, 2):
            qc.cz(int(perm[i]), int(perm[i + 1]))
    return qc.release()


def qft(n: int, basis_state: int | None = None) -> IRModule:
    """QFT|x> = 2^{-n/2} sum_k exp(2 pi i x k / 2^n) |k> (little endian):
    for i = n-1 .. 0: H(i), then CP(j, i, pi/2^(i-j)) for j = i-1 .. 0;
    finally SWAP(i, n-1-i).  `basis_state` prepends X gates preparing |x>."""
    qc = QuantumCircuit(n)
    if basis_state is not None:
        for q in range(n):
            if (basis_state >> q) & 1:
                qc.x(q)
    for i in range(n - 1, -1, -1):
        qc.h(i)
        for j in range(i - 1, -1, -1):
            qc.cp(j, i, math.pi / float(1 << (i - j)))
    for i in range(n // 2):
        qc.swap(i, n - 1 - i)
    return qc.release()


def qft_expected(n: int, x: int) -> np.ndarray:
    """Analytic QFT|x>: the phase index (x*k) mod 2^n is exact in integers."""
    k = np.arange(1 << n, dtype=np.uint64)
    ph = (np.uint64(x) * k) & np.uint64((1 << n) - 1)
    return np.exp(2j * np.pi * ph.astype(np.float64) / float(1 << n)) / math.sqrt(float(1 << n))


def hea(n: int, depth: int, seed: int) -> IRModule:
    """Hardware-efficient ansatz: per layer RY(theta), RZ(theta) on every
    qubit (theta~U[0,2pi)), then a CZ ladder CZ(i, i+1)."""
    rng = np.random.default_rng(seed)
    qc = QuantumCircuit(n)
    for _ in range(depth):
        th = rng.uniform(0.0, 2.0 * math.pi, size=(n, 2))
        for q in range(n):
            qc.ry(q, th[q, 0])
            qc.rz(q, th[q, 1])
        for i in range(n - 1):
            qc.cz(i, i + 1)
    return qc.release()


def hea_batch(count: int = 4096, seed: int = 2024, n_min: int = 10, n_max: int = 20,
              d_min: int = 8, d_max: int = 32) -> list[IRModule]:
    """`count` HEA circuits: n = round(exp(U[ln n_min, ln n_max])), depth
    ~ U{d_min..d_max}, angles from the same seeded stream."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=count))).astype(int)
    ds = rng.integers(d_min, d_max + 1, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [hea(int(n), int(d), int(sd)) for n, d, sd in zip(ns, ds, seeds)]


def serving_requests(count: int, seed: int = 7, n_min: int = 12, n_max: int = 30, d_min: int = 10,
                     d_max: int = 40) -> list[IRModule]:
    """The served workload: the H/RX + CX-ladder recipe of random_h_rx_cx
    with n = round(exp(U[ln n_min, ln n_max])) and `layers` ~ U{d_min..d_max}."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=count))).astype(int)
    ds = rng.integers(d_min, d_max + 1, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    return [random_h_rx_cx(int(n), int(d), int(sd)) for n, d, sd in zip(ns, ds, seeds)]


def poisson_arrivals(count: int, rate_hz: float, seed: int = 11) -> np.ndarray:
    """Arrival times (seconds) of a Poisson process with the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=count))


def expect_z_of(state: np.ndarray, n: int) -> np.ndarray:
    """<Z_q> = sum |a|^2 (1 - 2 bit_q) of a state vector (FP64)."""
    p = np.abs(np.asarray(state, dtype=np.complex128)) ** 2
    idx = np.arange(p.size, dtype=np.int64)
    return np.array([p.sum() - 2.0 * p[((idx >> q) & 1) == 1].sum() for q in range(n)])


def clustered(n: int, cluster: int = 6, depth: int = 15) -> IRModule:
    """bench_hw_awareness.cpp:30-53: per cluster of `cluster` qubits, `depth`
    times (H on each qubit, then a CX chain)."""
    qc = QuantumCircuit(n)
    for start in range(0, n, cluster):
        end = min(start + cluster, n)
        for _ in range(depth):
            for q in range(start, end):
                qc.h(q)
            for q in range(start, end - 1):
                qc.cx(q, q + 1)
    return qc.release()


def logical_gate_count(module: IRModule) -> int:
    """Gates that change the state (directives and barriers excluded)."""
    prog = module.program()
    t = prog["type"]
    return int(np.count_nonzero(t < 0xE0))


def to_reference_ir(module: IRModule) -> IRModule:
    """Rewrites the additive CZ / CP types as 2-qubit UNITARY diagonals, the
    form in which the reference engine can execute them."""
    prog = module.program()
    pool = UnitaryPool()
    src = module.unitaries()
    remap = {}
    for i in range(src.num_matrices()):
        off, n, k = src._meta[i]
        remap[i] = pool.store(src.data[off:off + n], k)
    out = np.array(prog, copy=True)
    cache = {}
    for i, g in enumerate(prog):
        t = int(g["type"])
        if t in (GateType.UNITARY, GateType.FUSED_BLOCK):
            out[i]["payload"] = remap[int(g["payload"])]
        elif t in (GateType.CZ, GateType.CP):
            if t == GateType.CZ:
                d = (1.0, 1.0, 1.0, -1.0)
                key = ("cz",)
            else:
                phi = float(np.array([g["payload"]], dtype=np.uint32).view(np.float32)[0])
                d = (1.0, 1.0, 1.0, complex(math.cos(phi), math.sin(phi)))
                key = ("cp", int(g["payload"]))
            if key not in cache:
                cache[key] = pool.store(np.diag(np.array(d, dtype=np.complex128)), 2)
            q = [int(g["qubits"][0]), int(g["qubits"][1])]
            out[i] = make_instr(GateType.UNITARY, q, matrix_idx=cache[key], uid=int(g["uid"]))
    m = IRModule(module.num_qubits, unitary_pool=pool)
    m.set_program(out)
    return m

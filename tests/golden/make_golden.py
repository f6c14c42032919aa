"""Generates tests/golden/reference_cases.npz by running the UNMODIFIED
reference engine and middle end (oracle/_ref, compiled from the reference's
own headers by oracle/Makefile) on small circuits.  Run it in a container
where the reference sources are mounted:

    python tests/golden/make_golden.py

Cases:
  kat_*       the programs of the reference's known-answer tests
              (tests/backend/test_engine_kernels.cpp:48-230,
               tests/backend/test_engine_measure.cpp:46-124,
               tests/integration/algos_no_optimization.cpp:18-160)
  zoo_*       seeded random circuits over every reference instruction type
  cfg0_*      the 40-layer H/RX/CX recipe at 10 qubits
  fuse_*      reference Middleware::transpile with gate fusion
              (middleware.hpp:526-753); expected state = reference run of the
              fused stream
  win_*       reference windowing (middleware.hpp:759-860) with small k_safe;
              expected state = reference run of the UNWINDOWED stream (the
              reference engine ignores GLOBAL_SWAP, cpu_openmp_engine.hpp:217-219)
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from __graft_entry__ import package  # noqa: E402

package()
from qlassical_b200 import circuits  # noqa: E402
from qlassical_b200.ir import GateType, IRModule, QuantumCircuit, make_instr  # noqa: E402
from oracle import oracle  # noqa: E402
import zoo  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz")


def prog_of(gates, n):
    m = IRModule(n)
    for g in gates:
        m.append(g)
    return m


def G(t, *q, param=0.0, midx=None):
    return make_instr(t, list(q), param, midx)


def kat_cases():
    T = GateType
    cases = {}
    # test_engine_kernels.cpp
    for name, t in (("x", T.X), ("h", T.H), ("y", T.Y)):
        cases[f"kat_{name}"] = (prog_of([G(t, 0)], 1), None, 0)
    cases["kat_z"] = (prog_of([G(T.X, 0), G(T.Z, 0)], 1), None, 0)
    cases["kat_s"] = (prog_of([G(T.X, 0), G(T.S, 0)], 1), None, 0)
    cases["kat_rx_pi"] = (prog_of([G(T.RX, 0, param=math.pi)], 1), None, 0)
    cases["kat_ry_pi2"] = (prog_of([G(T.RY, 0, param=math.pi / 2)], 1), None, 0)
    cases["kat_cx_c_gt_t"] = (prog_of([G(T.X, 2), G(T.CX, 2, 0)], 3), None, 0)
    cases["kat_cx_c_lt_t"] = (prog_of([G(T.X, 0), G(T.CX, 0, 2)], 3), None, 0)
    cases["kat_swap_fwd"] = (prog_of([G(T.X, 0), G(T.SWAP, 0, 2)], 3), None, 0)
    cases["kat_swap_bwd"] = (prog_of([G(T.X, 2), G(T.SWAP, 2, 0)], 3), None, 0)
    cases["kat_ccx"] = (prog_of([G(T.X, 0), G(T.X, 1), G(T.CCX, 1, 0, 2)], 3), None, 0)
    cases["kat_cswap"] = (prog_of([G(T.X, 0), G(T.X, 1), G(T.CSWAP, 1, 0, 2)], 3), None, 0)
    m = prog_of([G(T.X, 0)], 3)
    sw = np.zeros((4, 4), dtype=np.complex128)
    sw[0, 0] = sw[1, 2] = sw[2, 1] = sw[3, 3] = 1.0
    idx = m.unitaries().store(sw, 2)
    m.append(G(T.UNITARY, 0, 2, midx=idx))
    cases["kat_unitary_q0q2"] = (m, None, 0)
    cases["kat_kickback"] = (prog_of([G(T.H, 0), G(T.X, 1), G(T.H, 1), G(T.CX, 0, 1)], 2), None, 0)
    # test_engine_measure.cpp (seed 42) and a Bell pair
    cases["kat_measure_h"] = (prog_of([G(T.H, 0), G(T.MEASURE, 0)], 1), None, 42)
    cases["kat_bell_measure"] = (prog_of([G(T.H, 0), G(T.CX, 0, 1), G(T.MEASURE, 0), G(T.MEASURE, 1)], 2), None, 7)
    # algos_no_optimization.cpp: Deutsch from |10>, teleportation (seed 37)
    init = np.zeros(4, dtype=np.complex128)
    init[2] = 1.0
    for nm, extra in (("const0", []), ("const1", [G(T.X, 1)]), ("bal_x", [G(T.CX, 0, 1)]),
                      ("bal_notx", [G(T.CX, 0, 1), G(T.X, 0)])):
        cases[f"kat_deutsch_{nm}"] = (prog_of([G(T.H, 0), G(T.H, 1)] + extra + [G(T.H, 0)], 2), init, 37)
    tinit = np.zeros(8, dtype=np.complex128)
    tinit[0] = 1 / math.sqrt(3)
    tinit[1] = 1j * math.sqrt(2 / 3)
    cases["kat_teleport_alice"] = (prog_of([G(T.H, 1), G(T.CX, 1, 2), G(T.CX, 0, 1), G(T.H, 0),
                                            G(T.MEASURE, 0), G(T.MEASURE, 1)], 3), tinit, 37)
    return cases


def main():
    store = {}

    def put(name, module, init, seed, expected, meas):
        prog = module.program()
        store[f"{name}/n"] = np.array(module.num_qubits)
        store[f"{name}/prog"] = np.frombuffer(prog.tobytes(), dtype=np.uint8)
        store[f"{name}/pool_data"] = module.unitaries().data
        store[f"{name}/pool_meta"] = np.frombuffer(module.unitaries().metadata().tobytes(), dtype=np.uint8)
        store[f"{name}/init"] = init if init is not None else np.zeros(0, dtype=np.complex128)
        store[f"{name}/seed"] = np.array(seed)
        store[f"{name}/expected"] = expected
        store[f"{name}/meas"] = np.array(meas, dtype=np.uint8)

    for name, (m, init, seed) in kat_cases().items():
        st, meas = oracle.run_reference(m, init=init, seed=seed)
        put(name, m, init, seed, st, meas)

    for n in range(1, 11):
        for s in range(2):
            m = zoo.random_circuit(n, 12 * n + 8, seed=100 * n + s)
            st, meas = oracle.run_reference(m, seed=1)
            put(f"zoo_{n}_{s}", m, None, 1, st, meas)
    m = zoo.random_circuit(7, 60, seed=77)
    init = zoo.random_state(7, 5)
    st, _ = oracle.run_reference(m, init=init, seed=1)
    put("zoo_init_7", m, init, 1, st, [])

    m = circuits.random_h_rx_cx(10, 40, seed=2024)
    st, _ = oracle.run_reference(m, seed=1)
    put("cfg0_10", m, None, 1, st, [])

    for nm, m in (("kat_h_cx_x", None), ("clustered8", circuits.clustered(8, 4, 3)),
                  ("zoo8", zoo.random_circuit(8, 80, seed=8, types=["h", "x", "y", "z", "s", "cx", "u1", "u2"]))):
        if m is None:
            qc = QuantumCircuit(2)
            qc.h(0).cx(0, 1).x(1)
            m = qc.release()
        prog, data, meta = oracle.transpile_reference(m, fusion=True, hw=False)
        fused = zoo.module_from_arrays(m.num_qubits, prog, data, meta)
        st, _ = oracle.run_reference(fused, seed=1)
        put(f"fuse_{nm}", fused, None, 1, st, [])

    for nm, m, k_safe in (("tlb", None, 2), ("zoo10", zoo.random_circuit(10, 90, seed=10, types=[
            "h", "x", "y", "z", "s", "rx", "ry", "rz", "cx", "swap", "ccx", "cswap"]), 3)):
        if m is None:
            qc = QuantumCircuit(10)
            qc.x(0).x(1).cx(8, 9)
            m = qc.release()
        truth, _ = oracle.run_reference(m, seed=1)
        prog, data, meta = oracle.transpile_reference(m, fusion=False, hw=True, cost_model=1, k_safe=k_safe)
        win = zoo.module_from_arrays(m.num_qubits, prog, data, meta)
        put(f"win_{nm}", win, None, 1, truth, [])

    np.savez_compressed(OUT, **store)
    print(f"wrote {OUT}: {len([k for k in store if k.endswith('/n')])} cases")


if __name__ == "__main__":
    main()

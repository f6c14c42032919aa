"""The largest state one B200 holds: 34 qubits (137 GB complex64), on the
tile path with and without the tensor cores.  The circuit keeps <Z_i>
analytic: RY rotations (single gates and 5-qubit UNITARY blocks that are
Kronecker products of RY matrices, on low, middle and the highest qubits)
come first, then only diagonal gates (CZ, RZ), which leave <Z_i> unchanged,
so <Z_i> = cos(sum of the RY angles on qubit i).  Runs only on a GPU with
room for the state."""
import numpy as np
import pytest

N = 34


def _free_bytes():
    import ctypes
    from qlassical_b200 import _lib
    sm = ctypes.c_int()
    free = ctypes.c_uint64()
    total = ctypes.c_uint64()
    _lib.call("qlb_device_info", ctypes.byref(sm), ctypes.byref(free), ctypes.byref(total))
    return free.value


def _ry(t):
    c, s = np.cos(t / 2), np.sin(t / 2)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def _circuit(rng):
    from qlassical_b200.ir import QuantumCircuit
    qc = QuantumCircuit(N)
    total = np.zeros(N)
    for q in range(N):
        t = float(np.float32(rng.uniform(-np.pi, np.pi)))
        qc.ry(q, t)
        total[q] += t
    for qs in ([0, 1, 2, 3, 4], [5, 9, 17, 26, 33], [29, 30, 31, 32, 33], [2, 7, 12, 21, 30]):
        angles = rng.uniform(-1.0, 1.0, size=5)
        mat = np.array([[1.0]], dtype=np.complex128)
        for j in reversed(range(5)):          # matrix bit j <-> qs[j]
            mat = np.kron(mat, _ry(angles[j]))
        qc.unitary(qs, mat)
        total[qs] += angles
    for _ in range(40):
        a, b = rng.choice(N, size=2, replace=False)
        qc.cz(int(a), int(b))
    for q in range(0, N, 3):
        qc.rz(q, float(rng.uniform(-np.pi, np.pi)))
    return qc.release(), np.cos(total)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
def test_34_qubits_expect_z(mode):
    if _free_bytes() < (1 << N) * 8 + (4 << 30):
        pytest.skip("not enough free device memory for a 34-qubit state")
    import qlassical_b200 as q
    m, want = _circuit(np.random.default_rng(34))
    eng = q.CUDAEngine(N, mode=mode)
    eng.execute(m)
    assert abs(eng.norm_sq() - 1.0) < 1e-4
    got = eng.expect_z()
    assert np.abs(got - want).max() < 5e-5, np.abs(got - want).max()
    if mode == "tiled_tc":
        assert eng.last_stats()["tc_ops"] > 0
    del eng

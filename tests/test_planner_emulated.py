"""The tile planner checked on the CPU: its plan (qlb_describe_plan) is
replayed op by op in FP64 by tests/plan_emulator.py and compared with the
oracle.  This covers pass formation, register phases, qubit mapping, control
masks, phase encoding and tensor-core fusion without a GPU."""
import numpy as np
import pytest

from qlassical_b200 import circuits
from qlassical_b200.engine import describe_plan
from oracle import oracle
from plan_emulator import emulate
import zoo

TOL = {"tiled": 2e-5, "tiled_tc": 5e-5}


def check(module, mode, init=None, physical=False, **opts):
    plan = describe_plan(module, module.num_qubits, mode, physical_global_swap=physical, **opts)
    want, _ = oracle.run_oracle(module, init=init)
    got = emulate(plan, init=init)
    d = oracle.max_abs_diff(want, got)
    assert d < TOL[mode], d
    assert oracle.infidelity(want, got) < 1e-6
    return plan


@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
@pytest.mark.parametrize("n", [13, 14, 16])
def test_zoo_all_types(n, mode):
    m = zoo.random_circuit(n, 250, seed=n, types=zoo.REF_TYPES + zoo.EXT_TYPES, max_dense=5)
    check(m, mode)


@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
@pytest.mark.parametrize("tile_low", [4, 5, 6])
def test_fixed_low_tile_qubits(tile_low, mode):
    """QLB_OPT_TILE_LOW: memory qubits 0..tile_low-1 are in every tile of
    every pass (runs of 2^tile_low amplitudes), with the same results."""
    m = zoo.random_circuit(16, 200, seed=40 + tile_low, types=zoo.REF_TYPES + zoo.EXT_TYPES, max_dense=5)
    plan = check(m, mode, tile_low=tile_low, tc_chain=False)
    for p in plan["passes"]:
        assert p["tile_pos"][:tile_low] == list(range(tile_low))
        assert p["n_low"] >= tile_low
    h = circuits.hea(18, 12, 5)
    check(h, mode, tile_low=tile_low, tc_chain=False)


def test_tile_low_out_of_range_is_rejected():
    m = circuits.hea(14, 2, 1)
    for bad in (2, 7):
        with pytest.raises(ValueError):
            describe_plan(m, 14, "tiled", tile_low=bad)


@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
def test_rotation_cz_circuit_uses_tensor_cores(mode):
    m = circuits.random_rot_cz(16, 8, seed=2)
    plan = check(m, mode)
    if mode == "tiled_tc":
        assert plan["stats"]["tc_ops"] > 0
    else:
        assert plan["stats"]["tc_ops"] == 0


@pytest.mark.parametrize("mode", ["tiled", "tiled_tc"])
@pytest.mark.parametrize("physical", [False, True])
def test_windowed_stream(mode, physical):
    if not oracle.reference_available():
        pytest.skip("oracle/_ref not built")
    m = zoo.random_circuit(15, 150, seed=5, types=["h", "rx", "cx", "swap", "ccx", "cz", "u2"])
    prog, data, meta = oracle.transpile_reference(m, fusion=False, hw=True, cost_model=1, k_safe=4)
    win = zoo.module_from_arrays(15, prog, data, meta)
    plan = describe_plan(win, 15, mode, physical_global_swap=physical)
    want, _ = oracle.run_oracle(m)
    assert oracle.max_abs_diff(want, emulate(plan)) < TOL[mode]


def test_qft_plan():
    x = 0b1011011101
    plan = describe_plan(circuits.qft(14, basis_state=x), 14, "tiled")
    assert oracle.max_abs_diff(circuits.qft_expected(14, x), emulate(plan)) < 1e-5


def test_plain_mode_plan_is_one_step_per_instruction():
    m = circuits.random_h_rx_cx(14, 3, seed=1)
    plan = describe_plan(m, 14, "plain")
    assert len(plan["steps"]) == m.gate_count() and plan["stats"]["tile_passes"] == 0


def _a_word_offset(ph, kappa_perm, i):
    """Byte offset of tile-local amplitude i in the tensor-core A operand of
    phase `ph`: row t = thread index, K index 2 kappa(m) (+1 for the
    imaginary part), 128-byte rows with 16-byte chunks swizzled by t & 7."""
    t = sum(((i >> p) & 1) << j for j, p in enumerate(ph["thr_pos"]))
    m = sum(((i >> p) & 1) << j for j, p in enumerate(ph["reg_pos"]))
    kap = sum(((m >> j) & 1) << kappa_perm[j] for j in range(5))
    return t * 128 + (((kap >> 2) ^ (t & 7)) << 4) + (kap & 3) * 4


@pytest.mark.parametrize("n,depth,seed", [(16, 8, 2), (18, 12, 7), (20, 24, 1234)])
def test_tensor_core_phase_entry_offsets(n, depth, seed):
    """Phases entered straight from the previous phase's registers: the
    per-bit offsets (a_thr, a_reg) must send every amplitude to its word of
    the new phase's A operand, as the tensor-core op reads it."""
    from qlassical_b200.middleware import Middleware, TranspilerConfig
    m = Middleware().transpile(circuits.random_rot_cz(n, depth, seed=seed),
                               config=TranspilerConfig(max_fusion_qubits=5))
    plan = check(m, "tiled_tc")
    entries = 0
    for P in plan["passes"]:
        for k, ph in enumerate(P["phases"]):
            if not ph["flags"] & 1:
                continue
            entries += 1
            assert k > 0 and ph["ops"][0]["kind"] == 9
            prev = P["phases"][k - 1]
            perm = [(ph["ops"][0]["flags"] >> (3 * j)) & 7 for j in range(5)]
            assert sorted(perm) == list(range(5))
            seen = set()
            for t in range(256):
                base = 0
                for j in range(8):
                    if (t >> j) & 1:
                        base ^= ph["a_thr"][j]
                for r in range(32):
                    off = base
                    for j in range(5):
                        if (r >> j) & 1:
                            off ^= ph["a_reg"][j]
                    i = sum(((t >> j) & 1) << p for j, p in enumerate(prev["thr_pos"]))
                    i |= sum(((r >> j) & 1) << p for j, p in enumerate(prev["reg_pos"]))
                    assert off == _a_word_offset(ph, perm, i)
                    seen.add(off)
            assert len(seen) == 8192 and max(seen) < 32768
    assert entries > 0


@pytest.mark.parametrize("n,depth", [(14, 12), (16, 24)])
def test_chain_passes_of_the_fused_rotation_circuit(n, depth):
    """The benchmarked form (k <= 5 fusion + windowing) in tensor-core mode:
    most passes are chain passes (phases of one tensor-core op each), which
    the emulator replays with the chain kernel's byte-level data movement."""
    from qlassical_b200.middleware import Middleware, TranspilerConfig
    m = circuits.random_rot_cz(n, depth, seed=1234)
    f = Middleware().transpile(m, config=TranspilerConfig(max_fusion_qubits=5))
    plan = describe_plan(f, n, "tiled_tc")
    chain = sum(1 for P in plan["passes"] if P["features"] & 32)
    assert chain >= 1 and plan["stats"]["chain_passes"] == chain
    want, _ = oracle.run_oracle(m)
    got = emulate(plan)
    assert oracle.max_abs_diff(want, got) < TOL["tiled_tc"]
    assert oracle.infidelity(want, got) < 1e-6


def _ends_with_diagonals(n, seed, signs_only=True):
    """5-qubit unitaries on tile qubits, then diagonal gates that no later
    gate targets: CZs across out-of-tile and in-tile qubits (sign terms);
    with signs_only False also an RZ and a CP on out-of-tile qubits."""
    import qlassical_b200 as q
    rng = np.random.default_rng(seed)
    qc = q.QuantumCircuit(n)
    for _ in range(4):
        qc.unitary([int(x) for x in rng.permutation(13)[:5]], zoo.random_unitary(5, rng))
    qc.cz(n - 3, n - 1)
    qc.cz(3, n - 2)
    qc.cz(0, 1)
    if not signs_only:
        qc.rz(n - 2, 0.7)
        qc.cp(3, n - 1, 0.4)
    qc.cz(2, 5)
    return qc.release()


@pytest.mark.parametrize("n", [15, 17])
def test_post_terms_of_the_last_chain_pass(n):
    """CZs still deferred at the end of the circuit leave the last pass's
    phases (which stay chain phases) and become its post terms, applied as
    sign flips as the chain kernel stores the tile; with the chain kernel
    off, or with a non-sign term among them (RZ, CP on out-of-tile qubits),
    they are a diagonal op in the last phase instead."""
    m = _ends_with_diagonals(n, n)
    init = zoo.random_state(n, 4)
    plan = check(m, "tiled_tc", init=init)
    P = plan["passes"][-1]
    assert P["features"] & 32 and P["post_n"] >= 2, (P["features"], P["post_n"])
    off = check(m, "tiled_tc", init=init, tc_chain=False)
    assert all(Q["post_n"] == 0 for Q in off["passes"])
    mixed = check(_ends_with_diagonals(n, n, signs_only=False), "tiled_tc", init=init)
    assert all(Q["post_n"] == 0 for Q in mixed["passes"])
    # the fused rotation circuit's last pass carries its trailing CZs this way
    from qlassical_b200.middleware import Middleware, TranspilerConfig
    f = Middleware().transpile(circuits.random_rot_cz(16, 8, seed=1), config=TranspilerConfig(max_fusion_qubits=5))
    plan = check(f, "tiled_tc")
    assert plan["passes"][-1]["post_n"] >= 1


@pytest.mark.parametrize("chain", [True, False])
def test_diagonal_term_after_a_tensor_core_run(chain):
    """A CP between a register qubit of the run being fused for the tensor
    cores and a qubit outside it, followed by more gates on the run's qubits
    and then a gate on the CP's register qubit: the term must land after the
    run (chain mode marks it and flushes the run first; otherwise the run
    is emitted when the term arrives), and before that last gate."""
    import qlassical_b200 as q
    rng = np.random.default_rng(21)
    n = 15
    qc = q.QuantumCircuit(n)
    qc.unitary([0, 1, 2, 3, 4], zoo.random_unitary(5, rng))
    qc.cp(2, 14, 0.9)
    qc.ry(3, 0.4)
    qc.unitary([1, 3], zoo.random_unitary(2, rng))
    qc.h(2)
    qc.cz(4, 13)
    qc.rx(4, -0.3)
    m = qc.release()
    check(m, "tiled_tc", init=zoo.random_state(n, 6), tc_chain=chain)


def test_post_sign_terms_as_the_producers_apply_them():
    """The chain kernel's producers apply a sign term to piece i = lane +
    32 c (tile-local amplitudes L = 2 lane + 64 c and L + 1) of a tile from
    the term's tile-local mask (record word 6): live when the tile's
    out-of-tile bits and the lane's bits hold the mask's, then firing where
    64 c + 1 holds the rest (amplitude L + 1) and, if the mask has no bit 0,
    for amplitude L too.  Compared with the memory-index rule on every piece
    of several tiles."""
    from plan_emulator import post_terms
    n = 17
    m = _ends_with_diagonals(n, n)
    plan = describe_plan(m, n, "tiled_tc")
    P = plan["passes"][-1]
    assert 1 <= P["post_n"] <= 4
    words = np.array(plan["mats"], dtype=np.uint32)
    tp = P["tile_pos"]
    tilemem = sum(1 << q for q in tp)
    out_mem = [q for q in range(n) if not (tilemem >> q) & 1]
    lane = np.arange(32)[:, None]
    c = np.arange(128)[None, :]
    L0 = 2 * lane + 64 * c                                       # (32, 128)
    to_mem = lambda L: sum(((L >> j) & 1) << tp[j] for j in range(13))
    for i, (mask, p1, p0) in enumerate(post_terms(plan, P)):
        assert abs(p1 + 1) < 1e-6 and abs(p0 - 1) < 1e-6
        tl = int(words[2 * P["post_data"] + 8 * i + 6])
        assert to_mem(tl) == mask & tilemem
        for tile in range(1 << len(out_mem)):
            base = sum(((tile >> j) & 1) << q for j, q in enumerate(out_mem))
            gl = to_mem(2 * lane)
            live = ((mask & ~tilemem) & ~base) == 0
            live = live & (((tl & 0x3E) & ~(2 * lane)) == 0)      # (32, 1)
            need = tl & 0x1FC1
            hit1 = live & (((64 * c + 1) & need) == need)
            hit0 = hit1 & ((tl & 1) == 0)
            g = base | to_mem(L0)
            assert np.array_equal(hit0, (g & mask) == mask)
            assert np.array_equal(hit1, ((g | 1) & mask) == mask)


def test_chain_producer_piece_addressing():
    """The chain kernel's producer warps move 16-byte pieces: piece i =
    lane + 32 c of a tile holds tile-local amplitudes 2 i, 2 i + 1, at
    memory index (lane's bits 1..5 -> tile qubits 1..5) | rowoff[c] (c's
    bits -> tile qubits 6..12) (chain.cu).  Every piece of the 64 KB buffer
    is covered exactly once, from the memory index its tile-local index
    maps to; producer warp w of W takes the rows c = w, w + W, ..."""
    rng = np.random.default_rng(3)
    for warps in (3, 4, 4, 5):
        tp = [0, 1, 2] + sorted(int(x) for x in rng.choice(np.arange(3, 30), 10, replace=False))
        mem_of = lambda l: sum(1 << tp[j] for j in range(13) if (l >> j) & 1)   # noqa: E731
        rowoff = [sum(1 << tp[6 + i] for i in range(7) if (c >> i) & 1) for c in range(128)]
        seen = {}
        for pw in range(warps):
            for lane in range(32):
                gl = sum(1 << tp[1 + i] for i in range(5) if (lane >> i) & 1)
                for c in range(pw, 128, warps):
                    d = 16 * lane + 512 * c
                    assert d not in seen
                    seen[d] = gl | rowoff[c]
        assert len(seen) == 4096 and all(g == mem_of(d // 8) for d, g in seen.items())


def test_chain_staged_swizzle_round_trip():
    """The chain kernel stages the last op's result at 8-byte word
    l ^ fold4(l) and its producers read piece i (amplitudes 2i, 2i+1) from
    16-byte unit i ^ (F >> 1), halves swapped when F = fold4(2i) is odd
    (chain.cu).  Replayed: every piece comes back in order, and the stores
    of one warp instruction whose lanes cover the four residues mod 4 hit
    32 distinct banks over two wavefronts."""
    fold4 = lambda i: ((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 15   # noqa: E731
    words = {}
    for l in range(8192):
        a = l ^ fold4(l)
        assert a not in words
        words[a] = l
    for lane in range(32):
        for c in range(128):
            i = lane + 32 * c
            f = fold4(2 * lane) ^ fold4(64 * c)
            assert f == fold4(2 * i)
            u = i ^ (f >> 1)
            lo, hi = words[2 * u], words[2 * u + 1]
            if f & 1:
                lo, hi = hi, lo
            assert (lo, hi) == (2 * i, 2 * i + 1)
    # lanes on positions with residues 0..3 mod 4 (plus one more): conflict-free
    for lanes in ([0, 1, 2, 3, 7], [4, 9, 6, 11, 12], [8, 1, 10, 3, 2]):
        banks = {}
        for ln in range(32):
            l = sum(1 << lanes[b] for b in range(5) if (ln >> b) & 1) | (1 << 5 if 5 not in lanes else 0)
            a = l ^ fold4(l)
            banks.setdefault((2 * a) % 32, 0)
            banks[(2 * a) % 32] += 1
        assert max(banks.values()) <= 2

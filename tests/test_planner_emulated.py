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


def check(module, mode, init=None, physical=False):
    plan = describe_plan(module, module.num_qubits, mode, physical_global_swap=physical)
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


def test_chain_load_warp_addressing():
    """The chain kernel's load warp walks its 128 16-byte pieces per lane in
    Gray-code order, XOR-ing one memory bit and one buffer-offset bit per
    step (chain.cu).  Replayed here: every piece of the 64 KB buffer is
    written exactly once, at an offset inside the buffer, from the memory
    index its tile-local index maps to."""
    rng = np.random.default_rng(3)
    for _ in range(4):
        tp = [0, 1, 2] + sorted(int(x) for x in rng.choice(np.arange(3, 30), 10, replace=False))
        mem_of = lambda l: sum(1 << tp[j] for j in range(13) if (l >> j) & 1)   # noqa: E731
        hb = [1 << tp[6 + i] for i in range(7)]
        seen = {}
        for lane in range(32):
            gl = sum(1 << tp[1 + i] for i in range(5) if (lane >> i) & 1)
            g, d = gl, 16 * lane
            for hi in range(16):
                if hi:
                    bit = (hi & -hi).bit_length() - 1
                    g ^= hb[3 + bit]
                    d ^= 4096 << bit
                for lo in range(8):
                    if lo:
                        bit = 0 if lo & 1 else (1 if lo & 2 else 2)
                        g ^= hb[bit]
                        d ^= 512 << bit
                    assert 0 <= d < 65536 and d % 16 == 0 and d not in seen
                    seen[d] = g
                g ^= hb[2]
                d ^= 2048
        assert len(seen) == 4096
        for d, g in seen.items():
            assert g == mem_of(d // 8)


def _chain_geometry(tp, n):
    """chain.cu's chain_tensor_map(): dimensions at the tile's runs of
    consecutive memory qubits (at most 8 long), the first five boxed, the
    rest enumerated by copies."""
    runs, i = [], 0
    while i < 13:
        ln = 1
        while i + ln < 13 and ln < 8 and tp[i + ln] == tp[i] + ln:
            ln += 1
        runs.append((tp[i], ln))
        i += ln
    nd = min(len(runs), 5)
    lo = [runs[d][0] if d < nd else 64 for d in range(5)]
    dims, box, strides = [], [], []
    for d in range(5):
        if d < nd:
            hi = runs[d + 1][0] if d + 1 < nd else n
            dims.append(1 << (hi - runs[d][0]))
            box.append(1 << runs[d][1])
        else:
            dims.append(1)
            box.append(1)
        if d > 0:
            strides.append(8 << runs[d][0] if d < nd else 8 << n)
    rem = [runs[r][0] + k for r in range(nd, len(runs)) for k in range(runs[r][1])]
    boxed = sum(runs[d][1] for d in range(nd))
    return lo, dims, box, strides, rem, 8 << boxed


def test_chain_tma_geometry():
    """Every TMA box of every tile lands its amplitudes at their tile-order
    offsets, inside the tensor and the 64 KB buffer, with 16-byte-aligned
    starts (chain.cu: chain_tensor_map, tile_coords)."""
    rng = np.random.default_rng(11)
    for n in (14, 17, 20, 30, 34):
        for _ in range(6):
            others = sorted(int(x) for x in rng.choice(np.arange(3, n), 10, replace=False))
            tp = [0, 1, 2] + others
            lo, dims, box, strides, rem, box_bytes = _chain_geometry(tp, n)
            out = [q for q in range(n) if q not in tp]
            assert box_bytes * (1 << len(rem)) == 65536 and box[0] * 8 % 16 == 0
            assert all(st % 16 == 0 and st < 2 ** 40 for st in strides)
            assert all(b <= 256 and b <= dm for b, dm in zip(box, dims)) and all(dm < 2 ** 32 for dm in dims)
            mem_of = lambda l: sum(1 << tp[j] for j in range(13) if (l >> j) & 1)   # noqa: E731
            for tile in [0, 1, (1 << (n - 13)) - 1, int(rng.integers(0, 1 << (n - 13)))]:
                base = sum(1 << out[j] for j in range(len(out)) if (tile >> j) & 1)
                for cpy in range(1 << len(rem)):
                    c = [0] * 5
                    for j, q in enumerate(out):
                        if (tile >> j) & 1:
                            d = max(k for k in range(5) if lo[k] <= q)
                            c[d] |= 1 << (q - lo[d])
                    for i, q in enumerate(rem):
                        if (cpy >> i) & 1:
                            c[4] |= 1 << (q - lo[4])
                    assert all(c[d] + box[d] <= dims[d] for d in range(5)) and (c[0] * 8) % 16 == 0
                    # box element (i0..i4) -> tensor element -> memory index; smem offset in tile order
                    idx = np.indices(box[::-1]).reshape(5, -1)[::-1]       # i0 fastest
                    addr = (c[0] + idx[0]) * 8
                    for d in range(1, 5):
                        addr = addr + (c[d] + idx[d]) * strides[d - 1]
                    mem = addr // 8
                    smem_l = cpy * (box_bytes // 8) + np.arange(idx.shape[1])
                    want = np.array([base | mem_of(int(l)) for l in smem_l])
                    assert np.array_equal(mem, want)

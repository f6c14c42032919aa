"""CPU emulation of an engine plan (qlb_describe_plan JSON), for testing the
planner without a GPU.  Each op is applied to the full complex128 state with
the same meaning the tile kernel gives it: register bit j of a phase is memory
qubit tile_pos[reg_pos[j]]; ctrl_mem are memory-qubit controls.  Tensor-core
ops are decoded from their bf16 hi/lo B-operand image, so the emulation sees
the same split-precision unitary the tensor cores use."""
from __future__ import annotations

import numpy as np

TOP_U1, TOP_X, TOP_SWAP, TOP_U2, TOP_DENSE, TOP_U1R, TOP_RX, TOP_CPHASE, TOP_DENSE_TC = range(1, 10)
TOP_DIAG = 11
TOP_KRON = 12          # five real 2x2 factors, one per register bit (plus a continuation record, kind 0)
STEP_PASS, STEP_PLAIN, STEP_MEASURE, STEP_SWAP = range(4)
PASS_CHAIN = 32


def apply_k(st, n, qubits, mat, ctrl_mask=0):
    """Dense 2^k matrix on `qubits` (matrix bit j <-> qubits[j]) where all
    bits of ctrl_mask are set."""
    k = len(qubits)
    idx = np.arange(1 << n, dtype=np.int64)
    zero = np.ones(idx.shape, dtype=bool)
    for q in qubits:
        zero &= ((idx >> q) & 1) == 0
    zero &= (idx & ctrl_mask) == ctrl_mask
    base = idx[zero]
    offs = np.array([sum(((j >> b) & 1) << qubits[b] for b in range(k)) for j in range(1 << k)], dtype=np.int64)
    g = base[:, None] | offs[None, :]
    st[g] = st[g] @ np.asarray(mat).T


def emulate(plan, init=None):
    n = plan["n"]
    st = np.zeros(1 << n, dtype=np.complex128)
    if init is None:
        st[0] = 1.0
    else:
        st[:] = init
    words = np.array(plan["mats"], dtype=np.uint32)             # raw 32-bit words, 2 per float2 slot
    m2 = words.view(np.float32).astype(np.float64).reshape(-1, 2) if words.size else np.zeros((0, 2))
    mats = m2[:, 0] + 1j * m2[:, 1] if len(m2) else np.zeros(0, dtype=np.complex128)
    for step in plan["steps"]:
        kind = step["kind"]
        if kind == STEP_PASS and plan["passes"][step["index"]]["features"] & PASS_CHAIN:
            emulate_chain_pass(plan, plan["passes"][step["index"]], st, n)
            continue
        if kind == STEP_PASS:
            P = plan["passes"][step["index"]]
            assert P.get("post_n", 0) == 0, "post terms on a pass the general tile kernel runs"
            tp = P["tile_pos"]
            for ph in P["phases"]:
                mq = [tp[r] for r in ph["reg_pos"]]
                tq = [tp[r] for r in ph["thr_pos"]]
                for op in ph["ops"]:
                    cmask = int(op["ctrl_mem"])
                    for j in range(5):
                        if (op["ctrl_reg"] >> j) & 1:
                            cmask |= 1 << mq[j]
                    m = np.array(op["m"]).reshape(4, 2)
                    mc = m[:, 0] + 1j * m[:, 1]
                    kd = op["kind"]
                    if kd == 0:                   # a TOP_KRON op's continuation record
                        continue
                    if kd == TOP_KRON:
                        q = np.array(op["kron"]).reshape(5, 2, 2)
                        for j in range(5):
                            apply_k(st, n, [mq[j]], q[j])
                        continue
                    if kd == TOP_U1:
                        apply_k(st, n, [mq[op["r0"]]], mc.reshape(2, 2), cmask)
                    elif kd == TOP_U1R:
                        apply_k(st, n, [mq[op["r0"]]], m[:, 0].reshape(2, 2), cmask)
                    elif kd == TOP_RX:
                        c, s = m[0]
                        apply_k(st, n, [mq[op["r0"]]], np.array([[c, -1j * s], [-1j * s, c]]), cmask)
                    elif kd == TOP_X:
                        apply_k(st, n, [mq[op["r0"]]], np.array([[0, 1], [1, 0]]), cmask)
                    elif kd == TOP_SWAP:
                        sw = np.eye(4)[[0, 2, 1, 3]]
                        apply_k(st, n, [mq[op["r0"]], mq[op["r1"]]], sw, cmask)
                    elif kd == TOP_U2:
                        apply_k(st, n, [mq[op["r0"]], mq[op["r1"]]], mats[op["data"]:op["data"] + 16].reshape(4, 4),
                                cmask)
                    elif kd == TOP_DENSE:
                        k = op["k"]
                        D = 1 << k
                        apply_k(st, n, mq[:k], mats[op["data"]:op["data"] + D * D].reshape(D, D), cmask)
                    elif kd == TOP_DENSE_TC:
                        apply_k(st, n, mq[:5], decode_tc_flat(plan, op["data"], op["flags"]), 0)
                    elif kd == TOP_DIAG:
                        apply_diag(st, n, mq, op, words, tq)
                    elif kd == TOP_CPHASE:
                        idx = np.arange(1 << n, dtype=np.int64)
                        sel = (idx & cmask) == cmask
                        st[sel] *= mc[0]
                    else:
                        raise ValueError(f"unknown op kind {kd}")
        elif kind == STEP_PLAIN:
            t = step["type"]
            k = step["arity"]
            qs = step["qubits"][:max(k, 1)]
            if t in (0x80, 0xE0):
                D = 1 << k
                apply_k(st, n, qs[:k], mats[step["mat"]:step["mat"] + D * D].reshape(D, D))
            else:
                raise ValueError(f"plain step of type {t:#x} is not emulated")
        elif kind == STEP_SWAP:
            a, b = step["qubits"][:2]
            apply_k(st, n, [a, b], np.eye(4)[[0, 2, 1, 3]])
        else:
            raise ValueError("MEASURE steps are not emulated")
    return st


def apply_diag(st, n, mq, op, words, tq):
    """TOP_DIAG: R table over the register index, per-thread factor and sign
    tables over the thread index, T terms (thread/memory masks, p1 where all
    set else p0), S sign terms, G general mixed terms."""
    idx = np.arange(1 << n, dtype=np.int64)
    reg = np.zeros(idx.shape, dtype=np.int64)
    for j in range(5):
        reg |= ((idx >> mq[j]) & 1) << j
    thr = np.zeros(idx.shape, dtype=np.int64)
    for j in range(8):
        thr |= ((idx >> tq[j]) & 1) << j
    w = words[2 * op["data"]:].astype(np.uint64)
    f = words[2 * op["data"]:].view(np.float32).astype(np.float64)
    pos = 0
    fac = np.ones(idx.shape, dtype=np.complex128)
    if op["flags"] & 1:
        R = f[0:64:2] + 1j * f[1:64:2]
        fac *= R[reg]
        pos = 64
    if op["flags"] & 2:
        Tt = f[pos:pos + 512:2] + 1j * f[pos + 1:pos + 512:2]
        fac *= Tt[thr]
        pos += 512
    if op["flags"] & 4:
        St = w[pos:pos + 256].astype(np.int64)
        fac[((St[thr] >> reg) & 1) == 1] *= -1.0
        pos += 256
    n_gt = (op["flags"] >> 8) & 0xFF
    if n_gt:
        cms = [int(c) for c in w[pos:pos + n_gt]]
        pos += 4 * ((n_gt + 3) // 4)
        for k in range(n_gt):
            tab = f[pos:pos + 512:2] + 1j * f[pos + 1:pos + 512:2]
            hit = (reg & cms[k]) == cms[k]
            fac[hit] *= tab[thr[hit]]
            pos += 512
    n_t, n_s, n_g = op["n"] & 0xFFFF, op["n"] >> 16, op["ctrl_reg"]
    for _ in range(n_t):
        c = int(w[pos]) | (int(w[pos + 1]) << 32)
        p1 = f[pos + 2] + 1j * f[pos + 3]
        p0 = f[pos + 4] + 1j * f[pos + 5]
        on = (idx & c) == c
        fac *= np.where(on, p1, p0)
        pos += 8
    for _ in range(n_s):
        c = int(w[pos]) | (int(w[pos + 1]) << 32)
        pat = int(w[pos + 2])
        hit = ((idx & c) == c) & (((pat >> reg) & 1) == 1)
        fac[hit] *= -1.0
        pos += 4
    for _ in range(n_g):                      # groups: header {cm, count}, then count terms {mask, phase}
        cm, cnt = int(w[pos]), int(w[pos + 1])
        pos += 4
        for _ in range(cnt):
            c = int(w[pos]) | (int(w[pos + 1]) << 32)
            ph = f[pos + 2] + 1j * f[pos + 3]
            hit = ((idx & c) == c) & ((reg & cm) == cm)
            fac[hit] *= ph
            pos += 4
    st *= fac


def decode_tc_flat(plan, data, flags=None):
    """The split-precision unitary of a tensor-core op from its B image: row
    n = 2r + ro, column k = 2 kappa(c) + ri, kappa placing bit j of c at bit
    (flags >> 3j) & 7 (identity when flags is None).  Decoded matrices are
    cached in the plan dict itself (an id()-keyed global cache would hand a
    freed plan's matrices to a new plan that reuses its id)."""
    _tc_cache = plan.setdefault("_tc_cache", {})
    key = (data, flags)
    if key not in _tc_cache:
        flat = np.array(plan["mats"], dtype=np.uint32)    # raw words, 2 per float2 slot
        raw = flat[2 * data:2 * data + 4096].tobytes()
        u16 = np.frombuffer(raw, dtype=np.uint16).astype(np.uint32)
        nn = np.arange(64)[:, None]
        kk = np.arange(64)[None, :]
        at = (nn // 8) * 1024 + (kk // 8) * 128 + (nn % 8) * 16 + (kk % 8) * 2
        hi = (u16[at // 2] << 16).astype(np.uint32).view(np.float32).astype(np.float64)
        lo = (u16[(8192 + at) // 2] << 16).astype(np.uint32).view(np.float32).astype(np.float64)
        B = hi + lo
        perm = [j for j in range(5)] if flags is None else [(flags >> (3 * j)) & 7 for j in range(5)]
        kap = np.array([sum(((c >> j) & 1) << perm[j] for j in range(5)) for c in range(32)])
        _tc_cache[key] = B[0::2][:, 2 * kap] + 1j * B[1::2][:, 2 * kap]
    return _tc_cache[key]


def _tc_w(plan, data):
    """W[r][kap]: the complex matrix a tensor-core op's B image applies to
    the A row's amplitudes in K (kappa) order."""
    flat = np.array(plan["mats"], dtype=np.uint32)
    raw = flat[2 * data:2 * data + 4096].tobytes()
    u16 = np.frombuffer(raw, dtype=np.uint16).astype(np.uint32)
    nn = np.arange(64)[:, None]
    kk = np.arange(64)[None, :]
    at = (nn // 8) * 1024 + (kk // 8) * 128 + (nn % 8) * 16 + (kk % 8) * 2
    hi = (u16[at // 2] << 16).astype(np.uint32).view(np.float32).astype(np.float64)
    lo = (u16[(8192 + at) // 2] << 16).astype(np.uint32).view(np.float32).astype(np.float64)
    B = hi + lo
    return B[0::2][:, 0::2] + 1j * B[1::2][:, 0::2]


def _bits_or(idx, positions):
    """OR over the set bits j of idx of (1 << positions[j])."""
    out = np.zeros(np.shape(idx), dtype=np.int64)
    for j, p in enumerate(positions):
        out |= ((idx >> j) & 1) << int(p)
    return out


def _bits_xor(idx, values):
    out = np.zeros(np.shape(idx), dtype=np.int64)
    for j, v in enumerate(values):
        out ^= ((idx >> j) & 1) * int(v)
    return out


def emulate_chain_pass(plan, P, st, n):
    """The tensor-core chain kernel (chain.cu) replayed at byte level: the
    tile is read in phase 0's layout, scattered into the first op's A
    operand (own rows when phase 0 holds the op, else the entry offsets),
    multiplied by the op's B image, read back row by row and scattered into
    the next op's A by that phase's XOR offsets, and after the last op
    stored from the last phase's layout."""
    tp = P["tile_pos"]
    phases = P["phases"]
    first = 0 if phases[0]["ops"] else 1
    last = len(phases) - 1 if phases[-1]["ops"] else len(phases) - 2
    tile_set = set(tp)
    out_mem = [q for q in range(n) if q not in tile_set]
    t = np.arange(256, dtype=np.int64)[:, None]
    r = np.arange(32, dtype=np.int64)[None, :]
    R = phases[0]
    read_l = _bits_or(t, [R["thr_pos"][j] for j in range(8)]) | _bits_or(r, [R["reg_pos"][j] for j in range(5)])
    if first == 0:
        off0 = 128 * t + (((r // 4) ^ (t & 7)) << 4) + 4 * (r % 4)
    else:
        F = phases[first]
        off0 = _bits_xor(t, F["a_thr"]) ^ _bits_xor(r, F["a_reg"])
    l_all = np.arange(8192, dtype=np.int64)
    mem_l = _bits_or(l_all, tp)
    for tile in range(1 << (n - 13)):
        base = int(_bits_or(np.array(tile, dtype=np.int64), out_mem))
        buf = st[base | mem_l]
        v = buf[read_l]                              # (256, 32): thread t, register r
        off = off0
        for oi in range(first, last + 1):
            assert np.all(off % 4 == 0) and np.all(off < 32768) and np.unique(off).size == 8192
            row = off // 128
            chunk = ((off % 128) // 16) ^ (row & 7)
            kap = chunk * 4 + (off % 16) // 4
            A = np.zeros((256, 32), dtype=np.complex128)
            A[row, kap] = v
            W = _tc_w(plan, phases[oi]["ops"][0]["data"])
            v = A @ W.T                               # D row t, register r (phase oi's layout)
            if oi < last:
                F = phases[oi + 1]
                off = _bits_xor(t, F["a_thr"]) ^ _bits_xor(r, F["a_reg"])
        L = phases[last]
        g = base | _bits_or(t, [tp[p] for p in L["thr_pos"]]) | _bits_or(r, [tp[p] for p in L["reg_pos"]])
        st[g] = v
    apply_post_terms(plan, P, st, n)


def post_terms(plan, P):
    """The pass's post terms (TilePass::post_*): (memory mask, p1, p0) from
    32-byte records {u64 mask, float2 p1, float2 p0, pad} of the matrix buffer."""
    words = np.array(plan["mats"], dtype=np.uint32)
    out = []
    for i in range(P.get("post_n", 0)):
        w = words[2 * P["post_data"] + 8 * i: 2 * P["post_data"] + 8 * i + 8]
        f = w[2:6].view(np.float32).astype(np.float64)
        out.append((int(w[0]) | (int(w[1]) << 32), f[0] + 1j * f[1], f[2] + 1j * f[3]))
    return out


def apply_post_terms(plan, P, st, n):
    idx = np.arange(1 << n, dtype=np.int64)
    for mask, p1, p0 in post_terms(plan, P):
        st *= np.where((idx & mask) == mask, p1, p0)

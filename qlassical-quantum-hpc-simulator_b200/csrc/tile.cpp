// tile.cpp -- host planner: compiles an instruction stream into a plan.
//
// compile_plan() turns an instruction stream into a sequence of steps:
//   PASS  - one launch of the tile kernel (one HBM round trip) that applies
//           many instructions, split into register phases;
//   PLAIN - an instruction that runs outside tiles (MEASURE needs the host
//           RNG between its reduction and its collapse; a 6-qubit dense
//           block; a physical GLOBAL_SWAP).
// Pass formation scans the pending instructions in program order and takes
// every instruction whose register targets fit the 13-qubit tile and that
// does not depend on an instruction left behind (an instruction is only
// moved ahead of instructions that share no qubit with it, so the order of
// every pair of non-commuting instructions is preserved).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

#include "engine.h"
#include "kernels.h"
#include "plan.h"
#include "tile.h"

namespace qlb {

namespace {

constexpr uint64_t kLowMask = (uint64_t{1} << kLaneLow) - 1;  // memory qubits 0..4

struct Term {            // phase-polynomial term on memory qubits
    int a, b;            // -1 = absent
    uint32_t angle;      // turns * 2^32
};

struct MI {              // one instruction mapped to memory qubits
    uint8_t type = 0;
    uint32_t k = 0;
    uint32_t q[6] = {0, 0, 0, 0, 0, 0};
    uint64_t targets = 0;     // must be register qubits
    uint64_t ctrls = 0;       // control qubits (anywhere)
    uint64_t touched = 0;     // every qubit the instruction depends on
    bool diag = false;
    bool plain = false;       // runs as a PLAIN step (acts as a barrier)
    float param = 0.f;
    uint32_t matrix_idx = 0;
    std::vector<Term> terms;  // diag: its phase polynomial
    const qlb_gate_instr* src = nullptr;
};

uint32_t turns_u32(double rad) {
    double t = rad / (2.0 * M_PI);
    t -= std::floor(t);
    const double s = std::nearbyint(t * 4294967296.0);
    return static_cast<uint32_t>(static_cast<uint64_t>(s) & 0xFFFFFFFFull);
}

uint64_t bitm(uint32_t q) { return uint64_t{1} << q; }

// Diagonal UNITARY (k <= 2) with unit-modulus entries -> phase polynomial.
bool diag_terms(const qlb_pool_view* pool, const MI& mi, std::vector<Term>& out) {
    if (mi.k > 2) return false;
    const qlb_matrix_entry& e = pool->metadata[mi.matrix_idx];
    const double* d = pool->data + 2 * uint64_t{e.offset};
    const uint32_t D = 1u << mi.k;
    double arg[4];
    for (uint32_t r = 0; r < D; ++r)
        for (uint32_t c = 0; c < D; ++c) {
            const double re = d[2 * (r * D + c)], im = d[2 * (r * D + c) + 1];
            if (r != c) {
                if (re != 0.0 || im != 0.0) return false;
            } else {
                if (std::fabs(std::hypot(re, im) - 1.0) > 1e-9) return false;
                arg[r] = std::atan2(im, re);
            }
        }
    out.push_back({-1, -1, turns_u32(arg[0])});
    if (mi.k == 1) {
        out.push_back({static_cast<int>(mi.q[0]), -1, turns_u32(arg[1] - arg[0])});
    } else {
        out.push_back({static_cast<int>(mi.q[0]), -1, turns_u32(arg[1] - arg[0])});
        out.push_back({static_cast<int>(mi.q[1]), -1, turns_u32(arg[2] - arg[0])});
        out.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]),
                       turns_u32(arg[3] - arg[2] - arg[1] + arg[0])});
    }
    return true;
}

MI map_instr(const qlb_gate_instr& in, const Layout& lay, const qlb_pool_view* pool) {
    MI mi;
    mi.src = &in;
    mi.type = in.type;
    mi.param = in.payload.param;
    mi.matrix_idx = in.payload.matrix_idx;
    switch (in.type) {
    case QLB_H: case QLB_X: case QLB_Y: case QLB_Z: case QLB_S:
    case QLB_RX: case QLB_RY: case QLB_RZ: case QLB_MEASURE: mi.k = 1; break;
    case QLB_CX: case QLB_SWAP: case QLB_CZ: case QLB_CP: mi.k = 2; break;
    case QLB_CCX: case QLB_CSWAP: mi.k = 3; break;
    default: mi.k = in.flags_arity & 0x0F; break;
    }
    for (uint32_t j = 0; j < mi.k; ++j) {
        mi.q[j] = lay.mem[instr_qubit(in, j)];
        mi.touched |= bitm(mi.q[j]);
    }
    const double th = static_cast<double>(in.payload.param);
    switch (in.type) {
    case QLB_H: case QLB_Y: case QLB_RX: case QLB_RY: case QLB_X: mi.targets = bitm(mi.q[0]); break;
    case QLB_Z: mi.diag = true; mi.terms.push_back({static_cast<int>(mi.q[0]), -1, 0x80000000u}); break;
    case QLB_S: mi.diag = true; mi.terms.push_back({static_cast<int>(mi.q[0]), -1, 0x40000000u}); break;
    case QLB_RZ:
        mi.diag = true;
        mi.terms.push_back({-1, -1, turns_u32(-0.5 * th)});
        mi.terms.push_back({static_cast<int>(mi.q[0]), -1, turns_u32(th)});
        break;
    case QLB_CZ:
        mi.diag = true;
        mi.terms.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]), 0x80000000u});
        break;
    case QLB_CP:
        mi.diag = true;
        mi.terms.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]), turns_u32(th)});
        break;
    case QLB_CX: mi.targets = bitm(mi.q[1]); mi.ctrls = bitm(mi.q[0]); break;
    case QLB_CCX: mi.targets = bitm(mi.q[2]); mi.ctrls = bitm(mi.q[0]) | bitm(mi.q[1]); break;
    case QLB_SWAP: mi.targets = bitm(mi.q[0]) | bitm(mi.q[1]); break;
    case QLB_CSWAP: mi.targets = bitm(mi.q[1]) | bitm(mi.q[2]); mi.ctrls = bitm(mi.q[0]); break;
    case QLB_UNITARY: case QLB_FUSED_BLOCK:
        if (diag_terms(pool, mi, mi.terms)) {
            mi.diag = true;
        } else if (mi.k > static_cast<uint32_t>(kRegQubits)) {
            mi.plain = true;
        } else {
            for (uint32_t j = 0; j < mi.k; ++j) mi.targets |= bitm(mi.q[j]);
        }
        break;
    case QLB_MEASURE: mi.plain = true; break;
    default: break;
    }
    return mi;
}


// ---- phase building --------------------------------------------------------

struct PhaseBuild {
    std::vector<int> reg;            // tile-local positions, register bit order
    std::vector<uint32_t> ops;       // indices into the mapped stream
    int dense_k = 0;                 // 0 or the k of the DENSE op placed at bits 0..k-1
};

void choose_threads(const std::vector<int>& reg, bool edge, uint8_t* thr) {
    bool in_reg[kTileQubits] = {};
    for (int p : reg) in_reg[p] = true;
    std::vector<int> rest;
    for (int p = 0; p < kTileQubits; ++p)
        if (!in_reg[p]) rest.push_back(p);
    std::vector<int> order;
    if (edge) {
        order = rest;  // positions 0..4 first: lanes = memory qubits 0..4
    } else {
        // lanes 0..3 on positions with distinct residues mod 4 (conflict-free
        // half-warp shared-memory access under the XOR fold), then the rest
        std::vector<bool> used(rest.size(), false);
        for (int r = 0; r < 4; ++r)
            for (size_t i = 0; i < rest.size(); ++i)
                if (!used[i] && rest[i] % 4 == r) {
                    order.push_back(rest[i]);
                    used[i] = true;
                    break;
                }
        for (size_t i = 0; i < rest.size(); ++i)
            if (!used[i]) order.push_back(rest[i]);
    }
    for (int j = 0; j < kThreadQubits; ++j) thr[j] = static_cast<uint8_t>(order[j]);
}

void fill_reg(std::vector<int>& reg, bool edge) {
    bool in_reg[kTileQubits] = {};
    for (int p : reg) in_reg[p] = true;
    for (int p = (edge ? kLaneLow : 0); p < kTileQubits && static_cast<int>(reg.size()) < kRegQubits; ++p)
        if (!in_reg[p]) {
            reg.push_back(p);
            in_reg[p] = true;
        }
    for (int p = kTileQubits - 1; p >= 0 && static_cast<int>(reg.size()) < kRegQubits; --p)
        if (!in_reg[p]) {
            reg.push_back(p);
            in_reg[p] = true;
        }
}

class Planner {
public:
    Planner(qlb_engine& e, const qlb_pool_view* pool) : e_(e), pool_(pool), n_(e.sv.n) {}

    std::vector<MI> mi;
    TileProgram prog;
    std::vector<PlanStep> steps;
    qlb_exec_stats stats{};

    void plan(const qlb_gate_instr* in, uint64_t count) {
        if (e_.mode == QLB_MODE_TILED_TC) fail(QLB_ERR_INVALID_ARG, "tensor-core tiled mode is not available in this build");
        const bool tiled = e_.mode != QLB_MODE_PLAIN && n_ >= static_cast<uint32_t>(kTileQubits);
        Layout lay;
        lay.reset();
        uint32_t phys_to_log[64];
        for (uint32_t i = 0; i < 64; ++i) phys_to_log[i] = i;
        bool permuted = false;
        mi.reserve(count);
        for (uint64_t i = 0; i < count; ++i) {
            const qlb_gate_instr& g = in[i];
            if (g.type == QLB_BARRIER) continue;
            if (g.type == QLB_GLOBAL_SWAP) {
                const uint32_t p = g.qubits[0], v = g.qubits[1];
                if (p == v) continue;
                if (e_.physical_global_swap) {
                    // data moves: memory == physical layout; remember the owner
                    MI s;
                    s.type = QLB_GLOBAL_SWAP;
                    s.k = 2;
                    s.q[0] = p;
                    s.q[1] = v;
                    s.touched = bitm(p) | bitm(v);
                    s.src = &g;
                    s.plain = true;
                    mi.push_back(s);
                    std::swap(phys_to_log[p], phys_to_log[v]);
                    permuted = true;
                } else {
                    std::swap(lay.mem[p], lay.mem[v]);   // lazy: re-address later instructions
                }
                continue;
            }
            MI m = map_instr(g, lay, pool_);
            if (!tiled) m.plain = true;
            mi.push_back(std::move(m));
        }
        std::vector<uint32_t> pending(mi.size());
        for (uint32_t i = 0; i < pending.size(); ++i) pending[i] = i;
        while (!pending.empty()) {
            if (mi[pending[0]].plain) {
                emit_plain(mi[pending[0]]);
                pending.erase(pending.begin());
                continue;
            }
            std::vector<uint32_t> taken, rest;
            uint64_t T = kLowMask, blocked = 0;
            bool stop = false;
            for (uint32_t idx : pending) {
                const MI& m = mi[idx];
                if (stop || m.plain) {
                    stop = true;
                    rest.push_back(idx);
                    continue;
                }
                if (m.touched & blocked) {
                    blocked |= m.touched;
                    rest.push_back(idx);
                    continue;
                }
                const uint64_t nt = T | m.targets;
                if (__builtin_popcountll(nt) > kTileQubits) {
                    blocked |= m.touched;
                    rest.push_back(idx);
                    continue;
                }
                T = nt;
                taken.push_back(idx);
            }
            build_pass(T, taken);
            pending.swap(rest);
        }
        if (permuted) {
            // restore logical order: move logical L (now at physical p) back to bit L
            for (uint32_t L = 0; L < n_; ++L) {
                uint32_t p = L;
                while (phys_to_log[p] != L) ++p;
                if (p != L) {
                    emit_swap(p, L);
                    std::swap(phys_to_log[p], phys_to_log[L]);
                }
            }
        }
    }

    void emit_swap(uint32_t a, uint32_t b) {
        PlanStep st{};
        st.kind = STEP_SWAP;
        st.instr.qubits[0] = static_cast<uint8_t>(a);
        st.instr.qubits[1] = static_cast<uint8_t>(b);
        steps.push_back(st);
        stats.sweeps += 1;
        stats.permute_passes += 1;
        stats.launches += 1;
    }

    void emit_plain(const MI& m) {
        if (m.type == QLB_GLOBAL_SWAP) {
            emit_swap(m.q[0], m.q[1]);
            return;
        }
        PlanStep st{};
        st.instr = *m.src;
        for (uint32_t j = 0; j < m.k; ++j) {
            if (j < 4) st.instr.qubits[j] = static_cast<uint8_t>(m.q[j]);
            else st.instr.qubits_ext[j - 4] = static_cast<uint8_t>(m.q[j]);
        }
        if (m.type == QLB_MEASURE) {
            st.kind = STEP_MEASURE;
            stats.sweeps += 2;      // P(1) reduction + collapse
            stats.launches += 3;
        } else {
            st.kind = STEP_PLAIN;
            if (m.type == QLB_UNITARY || m.type == QLB_FUSED_BLOCK) {
                st.mat_off = push_mat_from_pool(m.matrix_idx);
                stats.dense_ops += 1;
            }
            stats.sweeps += 1;
            stats.launches += 1;
        }
        steps.push_back(st);
    }

private:
    qlb_engine& e_;
    const qlb_pool_view* pool_;
    uint32_t n_;

    void build_pass(uint64_t T, const std::vector<uint32_t>& ops) {
        // fill the tile with the lowest unused memory qubits
        for (uint32_t q = 0; q < n_ && __builtin_popcountll(T) < kTileQubits; ++q) T |= bitm(q);
        TilePass P{};
        int local_of[64];
        std::fill(local_of, local_of + 64, -1);
        int j = 0;
        for (uint32_t q = 0; q < n_; ++q) {
            if (T & bitm(q)) {
                P.tile_pos[j] = static_cast<uint8_t>(q);
                local_of[q] = j++;
            } else {
                P.out_mem[P.n_out++] = static_cast<uint8_t>(q);
            }
        }
        // register phases
        std::vector<PhaseBuild> phases;
        std::vector<uint32_t> rem = ops;
        bool first = true;
        while (!rem.empty()) {
            PhaseBuild pb;
            std::vector<uint32_t> later;
            uint64_t blocked = 0;
            std::vector<int> dense_q;   // ordered local positions of the phase's DENSE op
            for (uint32_t idx : rem) {
                const MI& m = mi[idx];
                if (m.touched & blocked) {
                    blocked |= m.touched;
                    later.push_back(idx);
                    continue;
                }
                std::vector<int> tl;
                for (uint32_t b = 0; b < n_; ++b)
                    if (m.targets & bitm(b)) tl.push_back(local_of[b]);
                bool ok = true;
                if (first)
                    for (int p : tl) ok = ok && p >= kLaneLow;
                const bool dense = !m.diag && m.k >= 3 && (m.type == QLB_UNITARY || m.type == QLB_FUSED_BLOCK);
                std::vector<int> mdq;
                if (dense) {
                    for (uint32_t jj = 0; jj < m.k; ++jj) mdq.push_back(local_of[m.q[jj]]);
                    if (!dense_q.empty() && dense_q != mdq) ok = false;
                }
                std::vector<int> nr = pb.reg;
                for (int p : tl)
                    if (std::find(nr.begin(), nr.end(), p) == nr.end()) nr.push_back(p);
                if (static_cast<int>(nr.size()) > kRegQubits) ok = false;
                if (!ok) {
                    blocked |= m.touched;
                    later.push_back(idx);
                    continue;
                }
                pb.reg = nr;
                if (dense) dense_q = mdq;
                pb.ops.push_back(idx);
            }
            if (pb.ops.empty() && first) {
                first = false;
                phases.push_back(PhaseBuild{});  // load-only phase
                continue;
            }
            if (!dense_q.empty()) {  // DENSE qubits occupy register bits 0..k-1 in matrix order
                std::vector<int> r = dense_q;
                for (int p : pb.reg)
                    if (std::find(r.begin(), r.end(), p) == r.end()) r.push_back(p);
                pb.reg = r;
                pb.dense_k = static_cast<int>(dense_q.size());
            }
            phases.push_back(pb);
            rem.swap(later);
            first = false;
        }
        if (phases.empty()) phases.push_back(PhaseBuild{});
        {
            bool low = false;
            for (int p : phases.back().reg) low = low || p < kLaneLow;
            if (low) phases.push_back(PhaseBuild{});  // store phase with lanes on qubits 0..4
        }
        P.phase_begin = static_cast<uint32_t>(prog.phases.size());
        for (size_t pi = 0; pi < phases.size(); ++pi) {
            PhaseBuild& pb = phases[pi];
            const bool edge = (pi == 0) || (pi + 1 == phases.size());
            fill_reg(pb.reg, edge);
            TilePhase ph{};
            for (int r = 0; r < kRegQubits; ++r) ph.reg_pos[r] = static_cast<uint8_t>(pb.reg[r]);
            choose_threads(pb.reg, edge, ph.thr_pos);
            ph.op_begin = static_cast<uint32_t>(prog.ops.size());
            encode_ops(pb, P, local_of);
            ph.op_end = static_cast<uint32_t>(prog.ops.size());
            prog.phases.push_back(ph);
        }
        P.phase_end = static_cast<uint32_t>(prog.phases.size());
        PlanStep st{};
        st.kind = STEP_PASS;
        st.index = static_cast<uint32_t>(prog.passes.size());
        steps.push_back(st);
        prog.passes.push_back(P);
        stats.tile_passes += 1;
        stats.sweeps += 1;
        stats.launches += 1;
    }

    int reg_bit(const PhaseBuild& pb, const int* local_of, uint32_t memq) const {
        const int l = local_of[memq];
        if (l < 0) return -1;
        for (int r = 0; r < kRegQubits; ++r)
            if (pb.reg[r] == l) return r;
        return -1;
    }

    uint32_t push_mat_from_pool(uint32_t matrix_idx) {
        const qlb_matrix_entry& e = pool_->metadata[matrix_idx];
        const double* d = pool_->data + 2 * uint64_t{e.offset};
        const uint32_t off = static_cast<uint32_t>(prog.mats.size());
        for (uint32_t i = 0; i < e.num_elements; ++i)
            prog.mats.push_back(make_float2(static_cast<float>(d[2 * i]), static_cast<float>(d[2 * i + 1])));
        if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
        return off;
    }

    void encode_ops(const PhaseBuild& pb, const TilePass&, const int* local_of) {
        std::vector<Term> run;  // consecutive diagonal instructions merged into one TOP_PHASE
        auto flush = [&]() {
            if (!run.empty()) encode_phase(pb, local_of, run);
            run.clear();
        };
        for (uint32_t idx : pb.ops) {
            const MI& m = mi[idx];
            if (m.diag) {
                run.insert(run.end(), m.terms.begin(), m.terms.end());
                continue;
            }
            flush();
            TileOp op{};
            for (uint32_t b = 0; b < n_; ++b) {
                if (!(m.ctrls & bitm(b))) continue;
                const int r = reg_bit(pb, local_of, b);
                if (r >= 0) op.ctrl_reg |= 1u << r;
                else op.ctrl_mem |= bitm(b);
            }
            switch (m.type) {
            case QLB_H: case QLB_Y: case QLB_RX: case QLB_RY: {
                op.kind = TOP_U1;
                op.r0 = static_cast<uint8_t>(reg_bit(pb, local_of, m.q[0]));
                Mat2f g = gate_matrix_1q(m.type, m.param);
                for (int i = 0; i < 4; ++i) op.m[i] = g.m[i];
                break;
            }
            case QLB_X:
                op.kind = TOP_X;
                op.r0 = static_cast<uint8_t>(reg_bit(pb, local_of, m.q[0]));
                break;
            case QLB_CX:
                op.kind = TOP_X;
                op.r0 = static_cast<uint8_t>(reg_bit(pb, local_of, m.q[1]));
                break;
            case QLB_CCX:
                op.kind = TOP_X;
                op.r0 = static_cast<uint8_t>(reg_bit(pb, local_of, m.q[2]));
                break;
            case QLB_SWAP: case QLB_CSWAP: {
                const uint32_t a = m.type == QLB_SWAP ? m.q[0] : m.q[1];
                const uint32_t b = m.type == QLB_SWAP ? m.q[1] : m.q[2];
                int ra = reg_bit(pb, local_of, a), rb = reg_bit(pb, local_of, b);
                if (ra > rb) std::swap(ra, rb);
                op.kind = TOP_SWAP;
                op.r0 = static_cast<uint8_t>(ra);
                op.r1 = static_cast<uint8_t>(rb);
                break;
            }
            default: {  // UNITARY / FUSED_BLOCK, non-diagonal, k <= 5
                const qlb_matrix_entry& e = pool_->metadata[m.matrix_idx];
                const double* d = pool_->data + 2 * uint64_t{e.offset};
                if (m.k == 1) {
                    op.kind = TOP_U1;
                    op.r0 = static_cast<uint8_t>(reg_bit(pb, local_of, m.q[0]));
                    for (int i = 0; i < 4; ++i)
                        op.m[i] = make_float2(static_cast<float>(d[2 * i]), static_cast<float>(d[2 * i + 1]));
                } else if (m.k == 2) {
                    int r0 = reg_bit(pb, local_of, m.q[0]), r1 = reg_bit(pb, local_of, m.q[1]);
                    op.kind = TOP_U2;
                    op.data = static_cast<uint32_t>(prog.mats.size());
                    // matrix bit 0 <-> q[0]; the kernel wants bit 0 <-> the lower register bit
                    const bool flip = r0 > r1;
                    for (int r = 0; r < 4; ++r)
                        for (int c = 0; c < 4; ++c) {
                            auto sw = [&](int x) { return flip ? (((x & 1) << 1) | ((x >> 1) & 1)) : x; };
                            const int src = sw(r) * 4 + sw(c);
                            prog.mats.push_back(make_float2(static_cast<float>(d[2 * src]),
                                                            static_cast<float>(d[2 * src + 1])));
                        }
                    if (flip) std::swap(r0, r1);
                    op.r0 = static_cast<uint8_t>(r0);
                    op.r1 = static_cast<uint8_t>(r1);
                } else {
                    op.kind = (e_.mode == QLB_MODE_TILED_TC && m.k == 5) ? TOP_DENSE_TC : TOP_DENSE;
                    op.k = static_cast<uint8_t>(m.k);
                    op.data = push_mat_from_pool(m.matrix_idx);
                    stats.dense_ops += 1;
                    if (op.kind == TOP_DENSE_TC) stats.tc_ops += 1;
                }
                break;
            }
            }
            prog.ops.push_back(op);
        }
        flush();
    }

    void encode_phase(const PhaseBuild& pb, const int* local_of, const std::vector<Term>& terms) {
        uint32_t hdr[kPhaseHeaderWords] = {};
        std::vector<uint32_t> thr, lin;
        auto pair_index = [](int j, int k) {
            if (j > k) std::swap(j, k);
            int idx = 0;
            for (int a = 0; a < kRegQubits; ++a)
                for (int b = a + 1; b < kRegQubits; ++b) {
                    if (a == j && b == k) return idx;
                    ++idx;
                }
            return -1;
        };
        for (const Term& t : terms) {
            if (t.a < 0) {
                hdr[0] += t.angle;
                continue;
            }
            const int ra = reg_bit(pb, local_of, static_cast<uint32_t>(t.a));
            const int rb = t.b >= 0 ? reg_bit(pb, local_of, static_cast<uint32_t>(t.b)) : -1;
            if (t.b < 0) {
                if (ra >= 0) hdr[1 + ra] += t.angle;
                else { thr.push_back(static_cast<uint32_t>(t.a) | (0xFFu << 8)); thr.push_back(t.angle); }
            } else if (ra >= 0 && rb >= 0) {
                hdr[6 + pair_index(ra, rb)] += t.angle;
            } else if (ra >= 0) {
                lin.push_back(static_cast<uint32_t>(ra) | (static_cast<uint32_t>(t.b) << 8));
                lin.push_back(t.angle);
            } else if (rb >= 0) {
                lin.push_back(static_cast<uint32_t>(rb) | (static_cast<uint32_t>(t.a) << 8));
                lin.push_back(t.angle);
            } else {
                thr.push_back(static_cast<uint32_t>(t.a) | (static_cast<uint32_t>(t.b) << 8));
                thr.push_back(t.angle);
            }
        }
        hdr[16] = static_cast<uint32_t>(thr.size() / 2);
        hdr[17] = static_cast<uint32_t>(lin.size() / 2);
        TileOp op{};
        op.kind = TOP_PHASE;
        op.data = static_cast<uint32_t>(prog.pdata.size());
        prog.pdata.insert(prog.pdata.end(), hdr, hdr + kPhaseHeaderWords);
        prog.pdata.insert(prog.pdata.end(), thr.begin(), thr.end());
        prog.pdata.insert(prog.pdata.end(), lin.begin(), lin.end());
        prog.ops.push_back(op);
    }
};

size_t align256(size_t x) { return (x + 255) & ~size_t{255}; }

}  // namespace

qlb_plan* compile_plan(qlb_engine& e, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool) {
    Planner pl(e, pool);
    pl.plan(prog, count);
    TileProgram& tp = pl.prog;
    auto* p = new qlb_plan();
    try {
        p->n = e.sv.n;
        p->mode = e.mode;
        p->steps = std::move(pl.steps);
        p->stats = pl.stats;
        p->stats.instructions = count;
        p->stats.sweep_bytes = static_cast<double>(p->stats.sweeps) * 16.0 * static_cast<double>(uint64_t{1} << e.sv.n);
        p->o_pass = 0;
        p->o_phase = align256(p->o_pass + tp.passes.size() * sizeof(TilePass));
        p->o_ops = align256(p->o_phase + tp.phases.size() * sizeof(TilePhase));
        p->o_pd = align256(p->o_ops + tp.ops.size() * sizeof(TileOp));
        p->o_mat = align256(p->o_pd + tp.pdata.size() * sizeof(uint32_t));
        const size_t total = align256(p->o_mat + tp.mats.size() * sizeof(float2));
        check_cuda(cudaStreamSynchronize(e.stream), "plan staging sync");
        char* h = static_cast<char*>(e.host_prog.ensure(total));
        std::memcpy(h + p->o_pass, tp.passes.data(), tp.passes.size() * sizeof(TilePass));
        std::memcpy(h + p->o_phase, tp.phases.data(), tp.phases.size() * sizeof(TilePhase));
        std::memcpy(h + p->o_ops, tp.ops.data(), tp.ops.size() * sizeof(TileOp));
        std::memcpy(h + p->o_pd, tp.pdata.data(), tp.pdata.size() * sizeof(uint32_t));
        std::memcpy(h + p->o_mat, tp.mats.data(), tp.mats.size() * sizeof(float2));
        void* d = p->dev.ensure(total);
        check_cuda(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, e.stream), "H2D plan");
    } catch (...) {
        delete p;
        throw;
    }
    return p;
}

void run_plan(qlb_engine& e, const qlb_plan& p) {
    if (p.n != e.sv.n) fail(QLB_ERR_INVALID_ARG, "plan was compiled for a different number of qubits");
    const char* d = static_cast<const char*>(p.dev.p);
    const float2* mats = reinterpret_cast<const float2*>(d + p.o_mat);
    for (const PlanStep& st : p.steps) {
        switch (st.kind) {
        case STEP_PASS:
            check_cuda(launch_tile_pass(e.sv.d, e.sv.n, reinterpret_cast<const TilePass*>(d + p.o_pass),
                                        reinterpret_cast<const TilePhase*>(d + p.o_phase),
                                        reinterpret_cast<const TileOp*>(d + p.o_ops),
                                        reinterpret_cast<const uint32_t*>(d + p.o_pd), mats, st.index, e.stream),
                       "tile pass");
            break;
        case STEP_PLAIN: apply_plain(e, st.instr, mats + st.mat_off); break;
        case STEP_MEASURE: measure(e, st.instr.qubits[0]); break;
        case STEP_SWAP: {
            const uint32_t a = st.instr.qubits[0], b = st.instr.qubits[1];
            uint32_t h[2] = {a, b};
            check_cuda(launch_swap_subspace(e.sv.d, e.sv.n, h, 2, uint64_t{1} << b, uint64_t{1} << a, e.stream),
                       "qubit swap");
            break;
        }
        default: break;
        }
    }
}

}  // namespace qlb

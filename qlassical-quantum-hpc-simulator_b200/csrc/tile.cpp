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
#include <complex>
#include <cstring>

#include "engine.h"
#include "kernels.h"
#include "plan.h"
#include "tile.h"

namespace qlb {

namespace {

struct Term {            // diagonal factor exp(i*angle) on amplitudes whose qubits a (and b) are 1
    int a, b;            // -1 = absent (a < 0: a global phase)
    double angle;        // radians
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

double wrap_angle(double rad) {           // to (-pi, pi]
    double t = std::fmod(rad, 2.0 * M_PI);
    if (t <= -M_PI) t += 2.0 * M_PI;
    if (t > M_PI) t -= 2.0 * M_PI;
    return t;
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
    out.push_back({-1, -1, (arg[0])});
    if (mi.k == 1) {
        out.push_back({static_cast<int>(mi.q[0]), -1, (arg[1] - arg[0])});
    } else {
        out.push_back({static_cast<int>(mi.q[0]), -1, (arg[1] - arg[0])});
        out.push_back({static_cast<int>(mi.q[1]), -1, (arg[2] - arg[0])});
        out.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]),
                       (arg[3] - arg[2] - arg[1] + arg[0])});
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
    case QLB_Z: mi.diag = true; mi.terms.push_back({static_cast<int>(mi.q[0]), -1, M_PI}); break;
    case QLB_S: mi.diag = true; mi.terms.push_back({static_cast<int>(mi.q[0]), -1, 0.5 * M_PI}); break;
    case QLB_RZ:
        mi.diag = true;
        mi.terms.push_back({-1, -1, (-0.5 * th)});
        mi.terms.push_back({static_cast<int>(mi.q[0]), -1, (th)});
        break;
    case QLB_CZ:
        mi.diag = true;
        mi.terms.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]), M_PI});
        break;
    case QLB_CP:
        mi.diag = true;
        mi.terms.push_back({static_cast<int>(mi.q[0]), static_cast<int>(mi.q[1]), (th)});
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
    uint64_t thr_mem[kThreadQubits] = {};   // memory qubit of thread bit j (set before encoding)
};

void choose_threads(const std::vector<int>& reg, bool edge, uint8_t* thr) {
    bool in_reg[kTileQubits] = {};
    for (int p : reg) in_reg[p] = true;
    std::vector<int> rest;
    for (int p = 0; p < kTileQubits; ++p)
        if (!in_reg[p]) rest.push_back(p);
    std::vector<int> order;
    if (edge) {
        order = rest;  // lowest free positions first: lanes on tile positions 0..4 where free
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

// ---- tensor-core phase entry ----------------------------------------------
// The A operand of a tensor-core op (128-byte swizzle, real and imaginary
// parts interleaved along K) puts the amplitude at tile-local index i at the
// XOR over i's set bits p of a_offset(p): register bit j of the phase is K
// bit kperm[j] (byte 4 << kperm[j]); thread bit j is row bit j (byte 128 << j,
// and for j < 3 the swizzle flips chunk bit j, byte 16 << j).
uint16_t a_offset(const TilePhase& ph, const int* kperm, int p) {
    for (int j = 0; j < kRegQubits; ++j)
        if (ph.reg_pos[j] == p) return static_cast<uint16_t>(4u << kperm[j]);
    for (int j = 0; j < kThreadQubits; ++j)
        if (ph.thr_pos[j] == p) return static_cast<uint16_t>((128u << j) ^ (j < 3 ? (16u << j) : 0u));
    return 0;
}

// Rank over GF(2) of the shared-memory bank bits (word address bits 0..4) of
// the previous phase's five lane positions: the 4-byte A stores of one warp
// instruction hit 2^(5 - rank) times the same bank.
int entry_bank_rank(const TilePhase& prev, const TilePhase& ph, const int* kperm) {
    uint32_t rows[5];
    for (int j = 0; j < 5; ++j) rows[j] = (a_offset(ph, kperm, prev.thr_pos[j]) >> 2) & 31u;
    int rank = 0;
    for (int bit = 4; bit >= 0; --bit) {
        int piv = -1;
        for (int j = rank; j < 5; ++j)
            if ((rows[j] >> bit) & 1u) {
                piv = j;
                break;
            }
        if (piv < 0) continue;
        std::swap(rows[rank], rows[piv]);
        for (int j = 0; j < 5; ++j)
            if (j != rank && ((rows[j] >> bit) & 1u)) rows[j] ^= rows[rank];
        ++rank;
    }
    return rank;
}

// The K permutation (of 120) with the fewest bank conflicts for the entry
// stores; the first found among equals, so the identity when it is as good.
void choose_kperm(const TilePhase& prev, const TilePhase& ph, int* kperm) {
    int p[kRegQubits] = {0, 1, 2, 3, 4};
    int best = -1;
    do {
        const int r = entry_bank_rank(prev, ph, p);
        if (r > best) {
            best = r;
            std::copy(p, p + kRegQubits, kperm);
            if (r == 5) break;
        }
    } while (std::next_permutation(p, p + kRegQubits));
}

// Thread order of a phase entered from the previous phase's registers: the
// previous lanes that become thread bits go to thread bits 0..2 (their rows
// flip distinct swizzle bits), from the highest of those slots down, leaving
// the low slots' banks to previous lanes that become register bits; the other
// lane slots take qubits the next phase holds in registers (so that entry
// has register-bound lanes too); then the rest in order.
void choose_threads_entry(const std::vector<int>& reg, const uint8_t* prev_thr, const std::vector<int>* next_reg,
                          uint8_t* thr) {
    bool in_reg[kTileQubits] = {}, used[kTileQubits] = {};
    for (int p : reg) in_reg[p] = true;
    int slot[kThreadQubits];
    std::fill(slot, slot + kThreadQubits, -1);
    std::vector<int> to_thr;
    int a = 0;
    for (int j = 0; j < 5; ++j) {
        if (in_reg[prev_thr[j]]) ++a;
        else to_thr.push_back(prev_thr[j]);
    }
    // slots 2, 1, 0 (bank bits 4, 3, 2) for up to three of them, the others at 3, 4, ...
    int s = 2, extra = 3;
    for (int p : to_thr) {
        int at;
        if (s >= 0 && s >= a - 2) at = s--;
        else at = extra++;
        slot[at] = p;
        used[p] = true;
    }
    std::vector<int> pref, rest;
    if (next_reg)
        for (int p : *next_reg)
            if (!in_reg[p] && !used[p]) pref.push_back(p);
    for (int p = 0; p < kTileQubits; ++p)
        if (!in_reg[p] && !used[p] && std::find(pref.begin(), pref.end(), p) == pref.end()) rest.push_back(p);
    std::vector<int> order = pref;
    order.insert(order.end(), rest.begin(), rest.end());
    // without a next entry to prepare, lanes 0..3 take distinct residues mod 4
    // where they can (conflict-free transposes under the XOR fold)
    bool res_used[4] = {};
    for (int j = 0; j < 4; ++j)
        if (slot[j] >= 0) res_used[slot[j] % 4] = true;
    for (int j = 0; j < kThreadQubits; ++j) {
        if (slot[j] >= 0) continue;
        size_t pick = 0;
        if (!next_reg && j < 4)
            for (size_t i = 0; i < order.size(); ++i)
                if (!res_used[order[i] % 4]) {
                    pick = i;
                    break;
                }
        slot[j] = order[pick];
        if (j < 4) res_used[slot[j] % 4] = true;
        order.erase(order.begin() + static_cast<long>(pick));
    }
    for (int j = 0; j < kThreadQubits; ++j) thr[j] = static_cast<uint8_t>(slot[j]);
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
    Planner(const PlanConfig& cfg, const qlb_pool_view* pool)
        : e_(cfg), pool_(pool), n_(cfg.n), low_mask_((uint64_t{1} << cfg.tile_low) - 1) {
        if (cfg.tile_low < kTileLow || cfg.tile_low > kTileLowMax)
            fail(QLB_ERR_INVALID_ARG, "tile_low must be in " + std::to_string(kTileLow) + ".." +
                                          std::to_string(kTileLowMax));
    }

    std::vector<MI> mi;
    TileProgram prog;
    std::vector<PlanStep> steps;
    qlb_exec_stats stats{};

    void plan(const qlb_gate_instr* in, uint64_t count) {
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
            const uint64_t T = pack_pass(pending, taken, rest);
            // deferred diagonal terms may ride into the next pass unless a
            // plain step (measurement, data permutation) or the end follows
            build_pass(T, taken, rest.empty() || mi[rest.front()].plain);
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

    // Chooses the instructions of the next pass from `pending` (program
    // order) and returns its tile qubits.  An instruction is ready when no
    // earlier instruction left out of the pass touches one of its qubits (it
    // then commutes with all of them); a plain step ends the window.  Ready
    // instructions whose targets are already tile qubits are taken at once;
    // otherwise the ready instruction adding the fewest new tile qubits is
    // taken (the earliest among equals), until none fits in 13.  The packing
    // kept is the best of several such greedy packings, each seeded with one
    // of the first ready instructions and scored (for streams of up to
    // kLookaheadMaxPending instructions) together with the best packing of
    // the pass after it.  Taken instructions keep their program order.
    uint64_t pack_pass(const std::vector<uint32_t>& pending, std::vector<uint32_t>& taken,
                       std::vector<uint32_t>& rest) {
        std::vector<char> in;
        // the look-ahead costs ~seeds^2 greedy packings: short streams only
        const uint64_t T = pack_best(pending, in, pending.size() <= kLookaheadMaxPending ? 1 : 0);
        for (size_t i = 0; i < pending.size(); ++i) (in[i] ? taken : rest).push_back(pending[i]);
        return T;
    }
    // Work of a packing: instructions plus 4 per target qubit.
    long pack_work(const std::vector<uint32_t>& pending, const std::vector<char>& in) const {
        long work = 0;
        for (size_t i = 0; i < in.size(); ++i)
            if (in[i]) work += 1 + 4 * __builtin_popcountll(mi[pending[i]].targets);
        return work;
    }
    // The packing of the next pass: the best of the greedy packings seeded
    // with each of the first ready instructions, scored by its own work plus
    // (depth > 0) the work of the best packing of the pass after it.
    static constexpr size_t kLookaheadMaxPending = 768;
    static constexpr size_t kSeeds = 12;
    uint64_t pack_best(const std::vector<uint32_t>& pending, std::vector<char>& best_in, int depth) {
        size_t window = pending.size();
        for (size_t i = 0; i < pending.size(); ++i)
            if (mi[pending[i]].plain) {
                window = i;
                break;
            }
        std::vector<int> seeds{-1};
        {
            uint64_t blocked = 0;
            for (size_t i = 0; i < window && seeds.size() < kSeeds; ++i) {
                const MI& m = mi[pending[i]];
                if (!(m.touched & blocked) && (m.targets & ~low_mask_)) seeds.push_back(static_cast<int>(i));
                blocked |= m.touched;
            }
        }
        uint64_t best_T = low_mask_;
        long best_score = -1;
        for (int seed : seeds) {
            std::vector<char> in(pending.size(), 0);
            uint64_t T = low_mask_;
            if (seed >= 0) {
                in[static_cast<size_t>(seed)] = 1;
                T |= mi[pending[static_cast<size_t>(seed)]].targets;
            }
            pack_greedy(pending, window, in, T);
            long score = pack_work(pending, in);
            if (depth > 0) {
                std::vector<uint32_t> rest;
                for (size_t i = 0; i < window; ++i)
                    if (!in[i]) rest.push_back(pending[i]);
                if (!rest.empty()) {
                    std::vector<char> in2;
                    pack_best(rest, in2, depth - 1);
                    score += pack_work(rest, in2);
                }
            }
            if (score > best_score) {
                best_score = score;
                best_in.swap(in);
                best_T = T;
            }
        }
        return best_T;
    }
    void pack_greedy(const std::vector<uint32_t>& pending, size_t window, std::vector<char>& in, uint64_t& T) {
        for (;;) {
            uint64_t blocked = 0;
            int best = -1, best_add = 64;
            for (size_t i = 0; i < window; ++i) {
                if (in[i]) continue;
                const MI& m = mi[pending[i]];
                if (m.touched & blocked) {
                    blocked |= m.touched;
                    continue;
                }
                const uint64_t nt = T | m.targets;
                const int add = __builtin_popcountll(nt & ~T);
                if (add == 0) {
                    in[i] = 1;
                    continue;
                }
                if (__builtin_popcountll(nt) <= kTileQubits && add < best_add) {
                    best = static_cast<int>(i);
                    best_add = add;
                }
                blocked |= m.touched;
            }
            if (best < 0) break;
            in[static_cast<size_t>(best)] = 1;
            T |= mi[pending[static_cast<size_t>(best)]].targets;
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
    PlanConfig e_;
    const qlb_pool_view* pool_;
    uint32_t n_;
    uint64_t low_mask_;   // memory qubits in every tile

    void build_pass(uint64_t T, const std::vector<uint32_t>& ops, bool final_pass) {
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
                // the first phase reads the tile as loaded: its lanes keep the
                // tile's low qubits 0..2 (runs of 8 amplitudes per 8 lanes)
                if (first)
                    for (int p : tl) ok = ok && p >= kTileLow;
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
            for (int p : phases.back().reg) low = low || p < kTileLow;
            if (low) phases.push_back(PhaseBuild{});  // store phase with lanes on tile positions 0..4
        }
        P.phase_begin = static_cast<uint32_t>(prog.phases.size());
        for (size_t pi = 0; pi < phases.size(); ++pi)
            fill_reg(phases[pi].reg, (pi == 0) || (pi + 1 == phases.size()));
        const bool tcm = e_.mode == QLB_MODE_TILED_TC;
        for (size_t pi = 0; pi < phases.size(); ++pi) {
            PhaseBuild& pb = phases[pi];
            const bool edge = (pi == 0) || (pi + 1 == phases.size());
            TilePhase ph{};
            for (int r = 0; r < kRegQubits; ++r) ph.reg_pos[r] = static_cast<uint8_t>(pb.reg[r]);
            // A phase that opens with a non-diagonal instruction in tensor-core
            // mode will likely open with its tensor-core op: it may be entered
            // straight from the previous phase's registers (kPhaseTcEntry).
            const bool cand = tcm && pi > 0 && !pb.ops.empty() && !mi[pb.ops[0]].diag;
            const TilePhase* prev = pi > 0 ? &prog.phases.back() : nullptr;
            if (cand && !edge) {
                // the next phase's registers, when it is itself an entry candidate
                const bool next_cand = pi + 1 < phases.size() && !phases[pi + 1].ops.empty() &&
                                       !mi[phases[pi + 1].ops[0]].diag;
                const std::vector<int>* next_reg = next_cand ? &phases[pi + 1].reg : nullptr;
                choose_threads_entry(pb.reg, prev->thr_pos, next_reg, ph.thr_pos);
            } else {
                choose_threads(pb.reg, edge, ph.thr_pos);
            }
            for (int j = 0; j < kThreadQubits; ++j) pb.thr_mem[j] = bitm(P.tile_pos[ph.thr_pos[j]]);
            ph.op_begin = static_cast<uint32_t>(prog.ops.size());
            if (cand) {
                choose_kperm(*prev, ph, entry_kperm_);
                entry_op_ = ph.op_begin;
            }
            phase_ops_begin_ = ph.op_begin;
            encode_ops(pb, P, local_of, final_pass && pi + 1 == phases.size());
            entry_op_ = ~0u;
            ph.op_end = static_cast<uint32_t>(prog.ops.size());
            if (cand && ph.op_end > ph.op_begin && prog.ops[ph.op_begin].kind == TOP_DENSE_TC) {
                ph.flags |= kPhaseTcEntry;
                for (int j = 0; j < kThreadQubits; ++j) ph.a_thr[j] = a_offset(ph, entry_kperm_, prev->thr_pos[j]);
                for (int j = 0; j < kRegQubits; ++j) ph.a_reg[j] = a_offset(ph, entry_kperm_, prev->reg_pos[j]);
            }
            prog.phases.push_back(ph);
        }
        P.phase_end = static_cast<uint32_t>(prog.phases.size());
        P.n_low = 0;
        while (P.n_low < kTileQubits && P.tile_pos[P.n_low] == P.n_low) ++P.n_low;
        const bool chain = chain_form(P);
        if (post_taken_) {
            if (chain) {
                emit_post(P);
            } else {
                for (const PTerm& x : post_terms_) add_pending(x.mask, x.p1, x.p0);
                flush_pending(phases.back(), local_of, nullptr, true);
                prog.phases.back().op_end = static_cast<uint32_t>(prog.ops.size());
            }
            post_terms_.clear();
            post_taken_ = false;
        }
        if (chain) {
            pass_features_ |= kPassChain;
            stats.chain_passes += 1;
        }
        P.features = static_cast<uint8_t>(pass_features_);
        // Every op must have a handler in the body the pass will run (a
        // missing one would be skipped by the kernel's dispatch).
        const int body = tile_body(pass_features_);
        for (uint32_t pi = P.phase_begin; pi < P.phase_end; ++pi)
            for (uint32_t oi = prog.phases[pi].op_begin; oi < prog.phases[pi].op_end; ++oi) {
                if (!tile_body_handles(body, prog.ops[oi].code))
                    fail(QLB_ERR_CUDA, "tile planner: op code " + std::to_string(prog.ops[oi].code) +
                                           " has no handler in kernel body " + std::to_string(body));
                if (prog.ops[oi].code == OPC_KRON) ++oi;     // its continuation record
            }
        PlanStep st{};
        st.kind = STEP_PASS;
        st.features = P.features;
        pass_features_ = 0;
        st.index = static_cast<uint32_t>(prog.passes.size());
        steps.push_back(st);
        prog.passes.push_back(P);
        stats.tile_passes += 1;
        stats.sweeps += 1;
        stats.launches += 1;
    }

    // A pass the tensor-core chain kernel can run: every register phase holds
    // exactly one op, a tensor-core op -- phase 0 (applied in its own layout,
    // identity K order) or an entry phase -- except an empty load phase
    // first and an empty store phase last.  Phase 0's entry offsets are
    // filled for its own layout so the chain kernel treats every op alike.
    bool chain_form(TilePass& P) {
        if (e_.mode != QLB_MODE_TILED_TC || !e_.tc_chain) return false;
        const uint32_t pb = P.phase_begin, pe = static_cast<uint32_t>(prog.phases.size());
        const uint32_t nph = pe - pb;
        if (nph == 0 || nph > kMaxSmemPhases) return false;
        auto nops = [&](uint32_t i) { return prog.phases[i].op_end - prog.phases[i].op_begin; };
        auto tc_only = [&](uint32_t i) { return nops(i) == 1 && prog.ops[prog.phases[i].op_begin].kind == TOP_DENSE_TC; };
        uint32_t first = pb;
        if (nops(pb) == 0) {
            first = pb + 1;
            if (first >= pe || !(prog.phases[first].flags & kPhaseTcEntry)) return false;
        }
        if (!tc_only(first)) return false;
        uint32_t last = first;
        for (uint32_t i = first + 1; i < pe; ++i) {
            if (nops(i) == 0 && i + 1 == pe) break;                 // store phase
            if (!tc_only(i) || !(prog.phases[i].flags & kPhaseTcEntry)) return false;
            last = i;
        }
        (void)last;
        if (first == pb) {
            static const int ident[kRegQubits] = {0, 1, 2, 3, 4};
            TilePhase& ph = prog.phases[pb];
            const uint32_t kp = prog.ops[ph.op_begin].flags;       // 3 bits per register bit
            for (int j = 0; j < kRegQubits; ++j)
                if (((kp >> (3 * j)) & 7u) != static_cast<uint32_t>(j)) return false;   // identity K order
            for (int j = 0; j < kThreadQubits; ++j) ph.a_thr[j] = a_offset(ph, ident, ph.thr_pos[j]);
            for (int j = 0; j < kRegQubits; ++j) ph.a_reg[j] = a_offset(ph, ident, ph.reg_pos[j]);
        }
        return true;
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

    // Accumulated global phase of the pass being built (constant terms of
    // RZ and diagonal UNITARYs); applied once at the end of its last phase.
    double pass_global_ = 0.0;
    int pass_features_ = 0;   // kPass* bits of the pass being built
    uint32_t phase_ops_begin_ = 0;   // first op of the phase being encoded
    // A tensor-core op emitted as op entry_op_ opens a kPhaseTcEntry
    // candidate phase and takes the K permutation entry_kperm_.
    uint32_t entry_op_ = ~0u;
    int entry_kperm_[kRegQubits] = {0, 1, 2, 3, 4};

    // ---- FP64 form of one register-level op --------------------------------
    using cd = std::complex<double>;
    struct HostOp {
        uint8_t kind = 0;
        int r0 = 0, r1 = 0, k = 0;
        uint32_t cm = 0;          // register control mask
        uint64_t cmem = 0;        // memory control mask (thread dependent)
        cd m[4];                  // 2x2 (row-major) or m[0] = phase
        std::vector<cd> mat;      // U2: 4x4 (bit 0 <-> r0 < r1); DENSE: 2^k x 2^k on bits 0..k-1
        double cost = 0.0;        // CUDA-core instructions per amplitude (planning estimate)
        bool diag = false;        // diagonal (a phase op), whatever its kind
    };

    std::vector<HostOp> host_ops(const PhaseBuild& pb, const int* local_of, const MI& m) {
        std::vector<HostOp> out;
        HostOp h;
        for (uint32_t b = 0; b < n_; ++b) {
            if (!(m.ctrls & bitm(b))) continue;
            const int r = reg_bit(pb, local_of, b);
            if (r >= 0) h.cm |= 1u << r;
            else h.cmem |= bitm(b);
        }
        const double r2 = 1.0 / std::sqrt(2.0), th = 0.5 * static_cast<double>(m.param);
        const cd I(0.0, 1.0);
        switch (m.type) {
        case QLB_H: h.kind = TOP_U1R; h.m[0] = r2; h.m[1] = r2; h.m[2] = r2; h.m[3] = -r2; h.cost = 2.5; break;
        case QLB_RY:
            h.kind = TOP_U1R; h.m[0] = std::cos(th); h.m[1] = -std::sin(th); h.m[2] = std::sin(th); h.m[3] = std::cos(th);
            h.cost = 2.5;
            break;
        case QLB_RX:
            h.kind = TOP_RX; h.m[0] = std::cos(th); h.m[1] = -I * std::sin(th); h.m[2] = -I * std::sin(th);
            h.m[3] = std::cos(th); h.cost = 2.5;
            break;
        case QLB_Y: h.kind = TOP_U1; h.m[0] = 0.0; h.m[1] = -I; h.m[2] = I; h.m[3] = 0.0; h.cost = 4; break;
        case QLB_X: case QLB_CX: case QLB_CCX:
            h.kind = TOP_X;
            h.m[0] = 0.0; h.m[1] = 1.0; h.m[2] = 1.0; h.m[3] = 0.0;
            h.cost = 0.5;
            break;
        case QLB_SWAP: case QLB_CSWAP: h.kind = TOP_SWAP; h.cost = 0.5; break;
        default: {
            const qlb_matrix_entry& e = pool_->metadata[m.matrix_idx];
            const cd* d = reinterpret_cast<const cd*>(pool_->data + 2 * uint64_t{e.offset});
            if (m.k == 1) {
                h.r0 = reg_bit(pb, local_of, m.q[0]);
                bool real = true;
                for (int i = 0; i < 4; ++i) {
                    h.m[i] = d[i];
                    real = real && d[i].imag() == 0.0;
                }
                h.kind = real ? TOP_U1R : TOP_U1;
                h.cost = real ? 2.5 : 4;
            } else if (m.k == 2) {
                int r0 = reg_bit(pb, local_of, m.q[0]), r1 = reg_bit(pb, local_of, m.q[1]);
                const bool flip = r0 > r1;
                h.kind = TOP_U2;
                h.mat.resize(16);
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c) {
                        auto sw = [&](int x) { return flip ? (((x & 1) << 1) | ((x >> 1) & 1)) : x; };
                        h.mat[r * 4 + c] = d[sw(r) * 4 + sw(c)];
                    }
                if (flip) std::swap(r0, r1);
                h.r0 = r0;
                h.r1 = r1;
                h.cost = 8;
            } else {
                h.kind = TOP_DENSE;
                h.k = static_cast<int>(m.k);
                h.mat.assign(d, d + e.num_elements);
                h.cost = 4.0 * static_cast<double>(1 << m.k);
            }
            out.push_back(std::move(h));
            return out;
        }
        }
        // 1- and 2-qubit standard gates: register targets
        if (m.type == QLB_SWAP || m.type == QLB_CSWAP) {
            const uint32_t a = m.type == QLB_SWAP ? m.q[0] : m.q[1];
            const uint32_t b = m.type == QLB_SWAP ? m.q[1] : m.q[2];
            int ra = reg_bit(pb, local_of, a), rb = reg_bit(pb, local_of, b);
            if (ra > rb) std::swap(ra, rb);
            h.r0 = ra;
            h.r1 = rb;
        } else {
            const uint32_t tq = (m.type == QLB_CX) ? m.q[1] : (m.type == QLB_CCX) ? m.q[2] : m.q[0];
            h.r0 = reg_bit(pb, local_of, tq);
        }
        out.push_back(std::move(h));
        return out;
    }

    // Applies a uniform (cmem == 0) op to one 5-qubit register vector.
    static void apply_host(const HostOp& h, cd* v) {
        const uint32_t cm = h.cm;
        auto ctl = [&](int i) { return (static_cast<uint32_t>(i) & cm) == cm; };
        switch (h.kind) {
        case TOP_U1: case TOP_U1R: case TOP_RX: case TOP_X:
            for (int i = 0; i < 32; ++i) {
                if (i & (1 << h.r0) || !ctl(i)) continue;
                const int j = i | (1 << h.r0);
                const cd a = v[i], b = v[j];
                v[i] = h.m[0] * a + h.m[1] * b;
                v[j] = h.m[2] * a + h.m[3] * b;
            }
            break;
        case TOP_SWAP:
            for (int i = 0; i < 32; ++i) {
                if (!(i & (1 << h.r0)) || (i & (1 << h.r1)) || !ctl(i)) continue;
                std::swap(v[i], v[i ^ (1 << h.r0) ^ (1 << h.r1)]);
            }
            break;
        case TOP_U2:
            for (int i = 0; i < 32; ++i) {
                if ((i & ((1 << h.r0) | (1 << h.r1))) || !ctl(i)) continue;
                const int idx[4] = {i, i | (1 << h.r0), i | (1 << h.r1), i | (1 << h.r0) | (1 << h.r1)};
                cd in[4], o[4];
                for (int c = 0; c < 4; ++c) in[c] = v[idx[c]];
                for (int r = 0; r < 4; ++r) {
                    o[r] = 0.0;
                    for (int c = 0; c < 4; ++c) o[r] += h.mat[r * 4 + c] * in[c];
                }
                for (int r = 0; r < 4; ++r) v[idx[r]] = o[r];
            }
            break;
        case TOP_DENSE: {
            const int D = 1 << h.k;
            for (int g = 0; g < 32; g += D) {
                cd o[32];
                for (int r = 0; r < D; ++r) {
                    o[r] = 0.0;
                    for (int c = 0; c < D; ++c) o[r] += h.mat[r * D + c] * v[g + c];
                }
                for (int r = 0; r < D; ++r) v[g + r] = o[r];
            }
            break;
        }
        case TOP_CPHASE:
            for (int i = 0; i < 32; ++i)
                if (ctl(i)) v[i] *= h.m[0];
            break;
        default: break;
        }
    }

    void emit_cuda_op(const HostOp& h) {
        TileOp op{};
        op.kind = h.kind;
        op.r0 = static_cast<uint8_t>(h.r0);
        op.r1 = static_cast<uint8_t>(h.r1);
        op.ctrl_reg = h.cm;
        op.ctrl_mem = h.cmem;
        op.has_mem = h.cmem != 0 ? 1 : 0;
        auto f2 = [](cd z) { return make_float2(static_cast<float>(z.real()), static_cast<float>(z.imag())); };
        const uint32_t r0 = static_cast<uint32_t>(h.r0);
        switch (h.kind) {
        case TOP_U1: case TOP_U1R: case TOP_RX:
            if (h.cm != 0) {                 // controlled: one complex handler for every 1-qubit kind
                op.kind = TOP_U1;
                op.code = static_cast<uint16_t>(OPC_U1_CTL + r0);
                for (int i = 0; i < 4; ++i) op.m[i] = f2(h.m[i]);
                pass_features_ |= kPassCtl;
            } else if (h.kind == TOP_U1) {
                op.code = static_cast<uint16_t>(OPC_U1 + r0);
                for (int i = 0; i < 4; ++i) op.m[i] = f2(h.m[i]);
            } else if (h.kind == TOP_U1R) {
                op.code = static_cast<uint16_t>(OPC_U1R + r0);
                for (int i = 0; i < 4; ++i) op.m[i] = make_float2(static_cast<float>(h.m[i].real()), 0.f);
            } else {
                op.code = static_cast<uint16_t>(OPC_RX + r0);
                op.m[0] = make_float2(static_cast<float>(h.m[0].real()), static_cast<float>(-h.m[1].imag()));
            }
            break;
        case TOP_X:
            op.code = static_cast<uint16_t>((h.cm != 0 ? OPC_X_CTL : OPC_X) + r0);
            pass_features_ |= kPassCtl;
            break;
        case TOP_SWAP:
            op.code = static_cast<uint16_t>(OPC_SWAP + reg_pair_index(r0, static_cast<uint32_t>(h.r1)));
            pass_features_ |= kPassSwaps;
            break;
        case TOP_CPHASE:
            op.code = OPC_CPHASE;
            op.m[0] = f2(h.m[0]);
            pass_features_ |= kPassCtl;
            break;
        case TOP_U2: case TOP_DENSE: {
            op.k = static_cast<uint8_t>(h.k);
            op.code = h.kind == TOP_U2 ? static_cast<uint16_t>(OPC_U2 + reg_pair_index(r0, static_cast<uint32_t>(h.r1)))
                      : h.k == 3       ? static_cast<uint16_t>(OPC_DENSE3)
                      : h.k == 4       ? static_cast<uint16_t>(OPC_DENSE4)
                                       : static_cast<uint16_t>(OPC_DENSE5);
            op.data = static_cast<uint32_t>(prog.mats.size());
            for (const cd& z : h.mat) prog.mats.push_back(f2(z));
            if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
            if (h.kind == TOP_DENSE) stats.dense_ops += 1;
            pass_features_ |= h.kind == TOP_U2 ? kPassPairs : kPassWide;
            break;
        }
        default: break;
        }
        prog.ops.push_back(op);
    }

    static uint16_t bf16_rn(float f) {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        u += 0x7FFFu + ((u >> 16) & 1u);
        return static_cast<uint16_t>(u >> 16);
    }
    static float bf16_f(uint16_t b) {
        const uint32_t u = static_cast<uint32_t>(b) << 16;
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }

    // B operand image (hi 8 KB + lo 8 KB, K-major canonical layout without
    // swizzle) of the real embedding of the 32x32 unitary U (row-major,
    // FP64): row n = 2 r + ro (output amplitude r, real / imaginary part),
    // column k = 2 kappa(c) + ri (input amplitude c, real / imaginary part),
    // kappa(c) placing bit j of c at bit kperm[j].  op.flags records kperm
    // (3 bits per register bit).
    void emit_tc_op(const std::vector<cd>& U, const int* kperm = nullptr) {
        static const int ident[kRegQubits] = {0, 1, 2, 3, 4};
        if (!kperm) kperm = ident;
        if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
        const uint32_t off = static_cast<uint32_t>(prog.mats.size());
        prog.mats.resize(prog.mats.size() + 2048, make_float2(0.f, 0.f));
        unsigned char* img = reinterpret_cast<unsigned char*>(prog.mats.data() + off);
        for (int c = 0; c < 32; ++c) {
            int kc = 0;
            for (int j = 0; j < kRegQubits; ++j)
                if ((c >> j) & 1) kc |= 1 << kperm[j];
            for (int n = 0; n < 64; ++n)
                for (int ri = 0; ri < 2; ++ri) {
                    const int r = n >> 1, ro = n & 1, kk = 2 * kc + ri;
                    const cd u = U[r * 32 + c];
                    const double x = ro == 0 ? (ri == 0 ? u.real() : -u.imag()) : (ri == 0 ? u.imag() : u.real());
                    const uint16_t hi = bf16_rn(static_cast<float>(x));
                    const uint16_t lo = bf16_rn(static_cast<float>(x - static_cast<double>(bf16_f(hi))));
                    const size_t at = static_cast<size_t>(n / 8) * 1024 + static_cast<size_t>(kk / 8) * 128 +
                                      static_cast<size_t>(n % 8) * 16 + static_cast<size_t>(kk % 8) * 2;
                    std::memcpy(img + at, &hi, 2);
                    std::memcpy(img + 8192 + at, &lo, 2);
                }
        }
        TileOp op{};
        op.kind = TOP_DENSE_TC;
        op.code = OPC_DENSE_TC;
        op.k = 5;
        op.data = off;
        for (int j = 0; j < kRegQubits; ++j) op.flags |= static_cast<uint32_t>(kperm[j]) << (3 * j);
        prog.ops.push_back(op);
        stats.dense_ops += 1;
        stats.tc_ops += 1;
        pass_features_ |= kPassTensorCores;
    }

    // Register-local ops waiting to be fused into one tensor-core op.
    struct Acc {
        std::vector<HostOp> ops;
        uint32_t touched = 0;   // register bits acted on non-diagonally
        double cost = 0.0;
    };

    // `whole_phase`: the run is everything the phase holds; with the chain
    // kernel on it goes to the tensor cores whatever its cost (the phase is
    // then a single tensor-core op, which a chain pass is made of).
    void flush(Acc& acc, bool whole_phase = false) {
        for (PTerm& t : pend_) t.after_acc = false;     // every pending term now follows the run
        if (acc.ops.empty()) return;
        if (acc.cost < e_.tc_min_cost && !(whole_phase && e_.tc_chain)) {   // cheaper as CUDA-core ops
            for (const HostOp& h : acc.ops) emit_cuda_op(h);
        } else {
            std::vector<cd> U(32 * 32, cd(0.0, 0.0));
            // A run that opens with a 5-qubit dense op (a fused block: its
            // matrix order is the register order) starts from that matrix
            // instead of simulating it on the 32 basis columns.
            size_t first = 0;
            if (acc.ops[0].kind == TOP_DENSE && acc.ops[0].k == 5 && acc.ops[0].cm == 0 && acc.ops[0].cmem == 0) {
                std::copy(acc.ops[0].mat.begin(), acc.ops[0].mat.end(), U.begin());
                first = 1;
            }
            for (int c = 0; c < 32; ++c) {
                cd col[32];
                for (int r = 0; r < 32; ++r) col[r] = first ? U[r * 32 + c] : ((r == c) ? cd(1.0, 0.0) : cd(0.0, 0.0));
                for (size_t i = first; i < acc.ops.size(); ++i) apply_host(acc.ops[i], col);
                for (int r = 0; r < 32; ++r) U[r * 32 + c] = col[r];
            }
            emit_tc_op(U, prog.ops.size() == entry_op_ ? entry_kperm_ : nullptr);
        }
        acc = Acc{};
    }

    static uint32_t nondiag_bits(const HostOp& h) {
        if (h.diag) return 0u;
        switch (h.kind) {
        case TOP_U1: case TOP_U1R: case TOP_RX: case TOP_X: return 1u << h.r0;
        case TOP_SWAP: case TOP_U2: return (1u << h.r0) | (1u << h.r1);
        case TOP_DENSE: return (1u << h.k) - 1u;
        default: return 0u;
        }
    }

    // ---- deferred diagonal terms --------------------------------------------
    // Diagonal gates commute with each other and with every gate whose
    // targets they do not touch.  Within a pass their phase terms are kept
    // (keyed by memory-qubit mask) and applied as one TOP_DIAG op only when
    // a later gate targets one of their qubits, or at the end of the pass.
    // A term multiplies amplitudes whose mask bits are all set by p1 and the
    // others by p0 (p0 != 1 only for single-qubit terms such as RZ).
    struct PTerm {
        uint64_t mask;
        cd p1, p0;
        bool after_acc = false;   // must follow the accumulator's current contents
    };
    std::vector<PTerm> pend_;
    uint64_t pend_qubits_ = 0;

    void add_pending(uint64_t mask, cd p1, cd p0, bool after_acc = false) {
        for (PTerm& t : pend_)
            if (t.mask == mask) {
                t.p1 *= p1;
                t.p0 *= p0;
                t.after_acc = t.after_acc || after_acc;
                return;
            }
        pend_.push_back({mask, p1, p0, after_acc});
        pend_qubits_ |= mask;
    }

    void split_mask(const PhaseBuild& pb, const int* local_of, uint64_t mask, uint32_t& cm, uint64_t& cmem) const {
        cm = 0;
        cmem = 0;
        for (uint64_t w = mask; w; w &= w - 1) {
            const uint32_t q = static_cast<uint32_t>(__builtin_ctzll(w));
            const int r = reg_bit(pb, local_of, q);
            if (r >= 0) cm |= 1u << r;
            else cmem |= bitm(q);
        }
    }

    // A register-only term as a (diagonal) accumulator op.
    static HostOp diag_host_op(uint32_t cm, cd p1, cd p0) {
        HostOp h;
        h.diag = true;
        if (std::abs(p0 - cd(1.0, 0.0)) < 1e-15) {
            h.kind = TOP_CPHASE;
            h.cm = cm;
            h.m[0] = p1;
            h.cost = 1.5;
        } else {                                   // single register bit, two phases
            h.kind = TOP_U1;
            h.r0 = __builtin_ctz(cm);
            h.m[0] = p0;
            h.m[1] = 0.0;
            h.m[2] = 0.0;
            h.m[3] = p1;
            h.cost = 4;
        }
        return h;
    }

    static bool is_one(cd z) { return std::abs(z - cd(1.0, 0.0)) < 1e-15; }

    // Emits the pending terms (and, when `global`, the pass's global phase)
    // as one TOP_DIAG op in phase `pb`.  With an accumulator (tensor-core
    // mode) register-only terms join it instead; every pending term commutes
    // with the accumulator's contents.
    std::vector<HostOp> rot_buf_;   // commuting 1-qubit rotations awaiting emission
    uint32_t rot_bits_ = 0;          // their register bits

    // Four or five real rotations (on distinct register bits) become one
    // TOP_KRON op: one dispatch for the run, identity on a missing bit.
    static constexpr int kKronMin = 4;
    void flush_rotations() {
        std::stable_sort(rot_buf_.begin(), rot_buf_.end(),
                         [](const HostOp& a, const HostOp& b) { return a.kind < b.kind; });
        int real = 0;
        for (const HostOp& h : rot_buf_) real += h.kind == TOP_U1R;
        for (const HostOp& h : rot_buf_)
            if (h.kind != TOP_U1R || real < kKronMin) emit_cuda_op(h);
        if (real >= kKronMin) emit_kron();
        rot_buf_.clear();
        rot_bits_ = 0;
    }
    void emit_kron() {
        float q[kRegQubits][4];
        for (int j = 0; j < kRegQubits; ++j) {
            q[j][0] = 1.f;
            q[j][1] = 0.f;
            q[j][2] = 0.f;
            q[j][3] = 1.f;
        }
        for (const HostOp& h : rot_buf_)
            if (h.kind == TOP_U1R)
                for (int i = 0; i < 4; ++i) q[h.r0][i] = static_cast<float>(h.m[i].real());
        TileOp op{}, cont{};
        op.kind = TOP_KRON;
        op.code = OPC_KRON;
        std::memcpy(&op.m[0], q[0], 16);
        std::memcpy(&op.m[2], q[1], 16);
        cont.code = OPC_NOP;
        std::memcpy(&cont.flags, q[2], 16);     // word 1: flags, n, ctrl_mem
        std::memcpy(&cont.m[0], q[3], 16);
        std::memcpy(&cont.m[2], q[4], 16);
        prog.ops.push_back(op);
        prog.ops.push_back(cont);
    }

    // Only the terms that share a qubit with `only` are emitted; the others
    // commute with the gate that caused the flush and stay pending.
    void flush_pending(const PhaseBuild& pb, const int* local_of, Acc* acc, bool global, uint64_t only = ~0ull) {
        cd R[32];
        for (cd& z : R) z = cd(1.0, 0.0);
        bool has_r = false;
        std::vector<PTerm> T;                                   // thread / memory-bit terms
        std::vector<std::pair<uint64_t, uint32_t>> S;           // mixed pi terms
        uint64_t thr_mask = 0;                                  // memory qubits on thread bits
        for (int j = 0; j < kThreadQubits; ++j) thr_mask |= pb.thr_mem[j];
        struct G {
            uint64_t cmem;
            uint32_t cm;
            cd p1;
        };
        std::vector<G> Gs;                                      // mixed general terms
        auto add_t = [&](uint64_t cmem, cd p1, cd p0) {
            for (PTerm& t : T)
                if (t.mask == cmem) {
                    t.p1 *= p1;
                    t.p0 *= p0;
                    return;
                }
            T.push_back({cmem, p1, p0});
        };
        // terms that came after a gate of the accumulated run on their
        // register bits are emitted after the run
        if (acc)
            for (const PTerm& t : pend_)
                if (t.after_acc && (t.mask & only)) {
                    flush(*acc);
                    break;
                }
        std::vector<PTerm> stay;
        for (const PTerm& t : pend_) {
            if (is_one(t.p1) && is_one(t.p0)) continue;
            if (!(t.mask & only)) {
                stay.push_back(t);
                continue;
            }
            uint32_t cm;
            uint64_t cmem;
            split_mask(pb, local_of, t.mask, cm, cmem);
            if (cmem == 0) {
                if (acc) {
                    HostOp h = diag_host_op(cm, t.p1, t.p0);
                    acc->cost += h.cost;
                    acc->ops.push_back(std::move(h));
                } else {
                    for (uint32_t m = 0; m < 32; ++m) R[m] *= ((m & cm) == cm) ? t.p1 : t.p0;
                    has_r = true;
                }
            } else if (cm == 0) {
                add_t(cmem, t.p1, t.p0);
            } else if (std::abs(t.p1 + cd(1.0, 0.0)) < 1e-12 && is_one(t.p0)) {
                uint32_t pat = 0;
                for (uint32_t m = 0; m < 32; ++m)
                    if ((m & cm) == cm) pat |= 1u << m;
                bool merged = false;
                for (auto& sterm : S)
                    if (sterm.first == cmem) {
                        sterm.second ^= pat;
                        merged = true;
                        break;
                    }
                if (!merged) S.emplace_back(cmem, pat);
            } else {
                Gs.push_back({cmem, cm, t.p1});
            }
        }
        pend_.swap(stay);
        pend_qubits_ = 0;
        for (const PTerm& t : pend_) pend_qubits_ |= t.mask;
        if (global) {
            const double g = wrap_angle(pass_global_);
            pass_global_ = 0.0;
            if (g != 0.0) {
                if (acc) {
                    HostOp h = diag_host_op(0u, std::polar(1.0, g), cd(1.0, 0.0));
                    acc->cost += h.cost;
                    acc->ops.push_back(std::move(h));
                } else {
                    add_t(0, std::polar(1.0, g), std::polar(1.0, g));
                }
            }
        }
        if (has_r) {                                     // a flat table is a scalar
            bool flat = true;
            for (uint32_t m = 1; m < 32; ++m) flat = flat && std::abs(R[m] - R[0]) < 1e-15;
            if (flat) {
                if (!is_one(R[0])) add_t(0, R[0], R[0]);
                has_r = false;
            }
        }
        T.erase(std::remove_if(T.begin(), T.end(), [](const PTerm& t) { return is_one(t.p1) && is_one(t.p0); }),
                T.end());
        S.erase(std::remove_if(S.begin(), S.end(), [](const auto& x) { return x.second == 0u; }), S.end());
        // Terms on thread bits only become per-thread tables (one load per
        // thread); terms touching out-of-tile qubits stay as lists.
        auto thread_bits = [&](uint32_t t) {
            uint64_t m = 0;
            for (int j = 0; j < kThreadQubits; ++j)
                if ((t >> j) & 1u) m |= pb.thr_mem[j];
            return m;
        };
        std::vector<cd> ttab;
        std::vector<uint32_t> stab;
        {
            std::vector<PTerm> keep;
            for (const PTerm& t : T) {
                if (t.mask != 0 && (t.mask & ~thr_mask) == 0) {
                    if (ttab.empty()) ttab.assign(256, cd(1.0, 0.0));
                    for (uint32_t th = 0; th < 256; ++th)
                        ttab[th] *= ((thread_bits(th) & t.mask) == t.mask) ? t.p1 : t.p0;
                } else {
                    keep.push_back(t);
                }
            }
            T.swap(keep);
            std::vector<std::pair<uint64_t, uint32_t>> skeep;
            for (const auto& x : S) {
                if ((x.first & ~thr_mask) == 0) {
                    if (stab.empty()) stab.assign(256, 0u);
                    for (uint32_t th = 0; th < 256; ++th)
                        if ((thread_bits(th) & x.first) == x.first) stab[th] ^= x.second;
                } else {
                    skeep.push_back(x);
                }
            }
            S.swap(skeep);
        }
        // General mixed terms on thread bits: one per-thread factor table per
        // distinct register mask (a CP between a register and a thread qubit).
        std::vector<uint32_t> gcm;
        std::vector<std::vector<cd>> gtab;
        {
            std::vector<G> gkeep;
            for (const G& g : Gs) {
                if ((g.cmem & ~thr_mask) != 0 || gcm.size() >= 255) {
                    gkeep.push_back(g);
                    continue;
                }
                size_t k = 0;
                while (k < gcm.size() && gcm[k] != g.cm) ++k;
                if (k == gcm.size()) {
                    gcm.push_back(g.cm);
                    gtab.emplace_back(256, cd(1.0, 0.0));
                }
                for (uint32_t th = 0; th < 256; ++th)
                    if ((thread_bits(th) & g.cmem) == g.cmem) gtab[k][th] *= g.p1;
            }
            Gs.swap(gkeep);
            std::stable_sort(Gs.begin(), Gs.end(), [](const G& a, const G& b) { return a.cm < b.cm; });
        }
        if (!has_r && ttab.empty() && stab.empty() && gcm.empty() && T.empty() && S.empty() && Gs.empty()) return;
        if (T.size() > 0xFFFF || S.size() > 0xFFFF) fail(QLB_ERR_INVALID_ARG, "too many diagonal terms in one pass");
        auto f2 = [](cd z) { return make_float2(static_cast<float>(z.real()), static_cast<float>(z.imag())); };
        auto words = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
            const uint32_t w[4] = {a, b, c, d};
            float2 f[2];
            std::memcpy(f, w, 16);
            prog.mats.push_back(f[0]);
            prog.mats.push_back(f[1]);
        };
        auto bits = [](float x) {
            uint32_t u;
            std::memcpy(&u, &x, 4);
            return u;
        };
        if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
        TileOp op{};
        op.kind = TOP_DIAG;
        op.code = OPC_DIAG;
        op.data = static_cast<uint32_t>(prog.mats.size());
        op.flags = (has_r ? 1u : 0u) | (ttab.empty() ? 0u : 2u) | (stab.empty() ? 0u : 4u) |
                   (static_cast<uint32_t>(gcm.size()) << 8);
        op.n = static_cast<uint32_t>(T.size()) | (static_cast<uint32_t>(S.size()) << 16);
        op.ctrl_reg = static_cast<uint32_t>(Gs.size());
        if (has_r)
            for (uint32_t m = 0; m < 32; ++m) prog.mats.push_back(f2(R[m]));
        for (const cd& z : ttab) prog.mats.push_back(f2(z));
        for (size_t th = 0; th < stab.size(); th += 2) {
            float2 f;
            std::memcpy(&f.x, &stab[th], 4);
            std::memcpy(&f.y, &stab[th + 1], 4);
            prog.mats.push_back(f);
        }
        for (size_t k = 0; k < gcm.size(); k += 4)    // register masks, four per 16 bytes
            words(gcm[k], k + 1 < gcm.size() ? gcm[k + 1] : 0u, k + 2 < gcm.size() ? gcm[k + 2] : 0u,
                  k + 3 < gcm.size() ? gcm[k + 3] : 0u);
        for (const auto& tab : gtab)
            for (const cd& z : tab) prog.mats.push_back(f2(z));
        for (const PTerm& t : T) {
            const float2 a = f2(t.p1), b = f2(t.p0);
            words(static_cast<uint32_t>(t.mask), static_cast<uint32_t>(t.mask >> 32), bits(a.x), bits(a.y));
            words(bits(b.x), bits(b.y), 0u, 0u);
        }
        for (const auto& x : S) words(static_cast<uint32_t>(x.first), static_cast<uint32_t>(x.first >> 32), x.second, 0u);
        // G terms by register mask (Gs is sorted by cm): a header {cm, count}
        // per group, then its terms {u64 mem mask, float2 phase}, 16 B each
        uint32_t n_groups = 0;
        for (size_t g = 0; g < Gs.size();) {
            size_t e = g;
            while (e < Gs.size() && Gs[e].cm == Gs[g].cm) ++e;
            words(Gs[g].cm, static_cast<uint32_t>(e - g), 0u, 0u);
            for (size_t k = g; k < e; ++k) {
                const float2 a = f2(Gs[k].p1);
                words(static_cast<uint32_t>(Gs[k].cmem), static_cast<uint32_t>(Gs[k].cmem >> 32), bits(a.x), bits(a.y));
            }
            ++n_groups;
            g = e;
        }
        op.ctrl_reg = n_groups;
        // Read from global memory, the op's tables and term lists cost a chain
        // of dependent L2 round trips (about one per table, per group and per
        // two T terms); when that chain is long the kernel first copies the
        // data (whole 16-byte words) into shared memory in one round trip and
        // two barriers.  m[0].x = the word count then, else 0.
        if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
        const uint32_t n_words = static_cast<uint32_t>((prog.mats.size() - op.data) / 2);
        const size_t chain = ((op.flags & 6u) ? 1 : 0) + (has_r ? 1 : 0) + gcm.size() + 2 * n_groups +
                             (T.size() + 1) / 2 + (S.size() + 3) / 4;
        const uint32_t stage_words = (chain >= 4 && n_words <= kDiagStageWords) ? n_words : 0u;
        std::memcpy(&op.m[0].x, &stage_words, 4);
        prog.ops.push_back(op);
    }

    void encode_ops(const PhaseBuild& pb, const TilePass&, const int* local_of, bool last_phase) {
        const bool tc = e_.mode == QLB_MODE_TILED_TC;
        Acc acc;
        for (uint32_t idx : pb.ops) {
            const MI& m = mi[idx];
            if (m.diag) {
                double g = 0.0;
                int singles = 0, others = 0;
                for (const Term& t : m.terms) {
                    if (t.a < 0) g += t.angle;
                    else if (t.b < 0) ++singles;
                    else ++others;
                }
                const bool fold = singles == 1 && others == 0;   // one qubit: the global part becomes p0
                if (!fold) pass_global_ += g;
                for (const Term& t : m.terms) {
                    if (t.a < 0) continue;
                    const uint64_t mask = bitm(static_cast<uint32_t>(t.a)) | (t.b >= 0 ? bitm(static_cast<uint32_t>(t.b)) : 0);
                    const cd p1 = std::polar(1.0, wrap_angle(fold ? g + t.angle : t.angle));
                    const cd p0 = fold ? std::polar(1.0, wrap_angle(g)) : cd(1.0, 0.0);
                    if (tc) {
                        uint32_t cm;
                        uint64_t cmem;
                        split_mask(pb, local_of, mask, cm, cmem);
                        if (cmem == 0) {                 // register-only: straight into the accumulator
                            HostOp h = diag_host_op(cm, p1, p0);
                            acc.cost += h.cost;
                            acc.ops.push_back(std::move(h));
                            continue;
                        }
                        // a term on register bits the run acts on must follow
                        // the run: with the chain kernel on it is marked so (a
                        // later flush emits it after the run, a post term
                        // follows everything), else the run is emitted now
                        if (cm & acc.touched) {
                            if (e_.tc_chain) {
                                add_pending(mask, p1, p0, true);
                                continue;
                            }
                            flush(acc);
                        }
                    }
                    add_pending(mask, p1, p0);
                }
                continue;
            }
            if (pend_qubits_ & m.targets) {
                flush_rotations();
                // tensor-core mode: only the terms on the gate's targets, so
                // the others can still join a later run or the post terms;
                // CUDA-core mode: all of them, in one op
                flush_pending(pb, local_of, tc ? &acc : nullptr, false, tc ? m.targets : ~0ull);
            }
            for (HostOp& h : host_ops(pb, local_of, m)) {
                if (!tc) {
                    // Uncontrolled 1-qubit rotations on distinct register bits
                    // commute: collect them and emit them grouped by kind, so
                    // the kernel sees long runs of one kind.
                    const bool rot = (h.kind == TOP_U1R || h.kind == TOP_RX || h.kind == TOP_U1) && h.cm == 0 &&
                                     h.cmem == 0;
                    if (rot && !(rot_bits_ & (1u << h.r0))) {
                        rot_bits_ |= 1u << h.r0;
                        rot_buf_.push_back(std::move(h));
                        continue;
                    }
                    flush_rotations();
                    if (rot) {
                        rot_bits_ |= 1u << h.r0;
                        rot_buf_.push_back(std::move(h));
                    } else {
                        emit_cuda_op(h);
                    }
                    continue;
                }
                if (h.cmem == 0) {                       // uniform over the tile: fusable
                    acc.touched |= nondiag_bits(h);
                    acc.cost += h.cost;
                    acc.ops.push_back(std::move(h));
                } else {
                    flush(acc);
                    emit_cuda_op(h);
                }
            }
        }
        flush_rotations();
        if (last_phase && !(tc && e_.tc_chain && take_post(pb, local_of, acc)))
            flush_pending(pb, local_of, tc ? &acc : nullptr, true);
        if (tc) flush(acc, prog.ops.size() == phase_ops_begin_);
    }

    // ---- post terms --------------------------------------------------------
    // At the end of a final pass in chain mode the deferred diagonal terms
    // leave the last phase, so that its tensor-core op stays alone in it: sign
    // terms (a CZ-like -1 where every mask bit is set, on any memory qubits)
    // become post terms, which the chain kernel applies as it stores the tile
    // (TilePass::post_*); register-only terms and the global phase join the
    // accumulated run.  If the pass does not run on the chain kernel after
    // all, the sign terms return as a TOP_DIAG op at the end of the last
    // phase (they commute with everything the phase applies after them).
    std::vector<PTerm> post_terms_;
    bool post_taken_ = false;

    bool take_post(const PhaseBuild& pb, const int* local_of, Acc& acc) {
        std::vector<PTerm> sign, reg;
        for (const PTerm& x : pend_) {
            if (is_one(x.p1) && is_one(x.p0)) continue;
            if (std::abs(x.p1 + cd(1.0, 0.0)) < 1e-12 && is_one(x.p0)) {
                sign.push_back(x);
                continue;
            }
            uint32_t cm;
            uint64_t cmem;
            split_mask(pb, local_of, x.mask, cm, cmem);
            if (cmem != 0) return false;
            reg.push_back(x);
        }
        if (sign.empty() || sign.size() > kPostMax) return false;
        for (const PTerm& x : reg) {
            uint32_t cm;
            uint64_t cmem;
            split_mask(pb, local_of, x.mask, cm, cmem);
            HostOp h = diag_host_op(cm, x.p1, x.p0);
            acc.cost += h.cost;
            acc.ops.push_back(std::move(h));
        }
        const double g = wrap_angle(pass_global_);
        if (g != 0.0) {
            HostOp h = diag_host_op(0u, std::polar(1.0, g), cd(1.0, 0.0));
            acc.cost += h.cost;
            acc.ops.push_back(std::move(h));
        }
        post_terms_.swap(sign);
        post_taken_ = true;
        pend_.clear();
        pend_qubits_ = 0;
        pass_global_ = 0.0;
        return true;
    }

    void emit_post(TilePass& P) {
        const std::vector<PTerm>& t = post_terms_;
        P.post_n = static_cast<uint32_t>(t.size());
        P.post_data = 0;
        if (t.empty()) return;
        if (prog.mats.size() & 1) prog.mats.push_back(make_float2(0.f, 0.f));
        P.post_data = static_cast<uint32_t>(prog.mats.size());
        for (const PTerm& x : t) {
            float2 w[4];
            std::memcpy(&w[0], &x.mask, 8);
            w[1] = make_float2(static_cast<float>(x.p1.real()), static_cast<float>(x.p1.imag()));
            w[2] = make_float2(static_cast<float>(x.p0.real()), static_cast<float>(x.p0.imag()));
            uint32_t tl[2] = {0u, 0u};
            for (int j = 0; j < kTileQubits; ++j)
                if (x.mask & bitm(P.tile_pos[j])) tl[0] |= 1u << j;
            std::memcpy(&w[3], tl, 8);
            for (const float2& f : w) prog.mats.push_back(f);
        }
    }
};

size_t align256(size_t x) { return (x + 255) & ~size_t{255}; }

}  // namespace

HostPlan plan_host(const PlanConfig& cfg, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool) {
    Planner pl(cfg, pool);
    pl.plan(prog, count);
    HostPlan h;
    h.steps = std::move(pl.steps);
    h.prog = std::move(pl.prog);
    h.stats = pl.stats;
    h.stats.instructions = count;
    return h;
}

qlb_plan* compile_plan(qlb_engine& e, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool,
                       DeviceBuffer* image) {
    Planner pl(PlanConfig{e.sv.n, e.mode, e.physical_global_swap, e.tc_min_cost, e.tc_chain, e.tile_low}, pool);
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
        p->o_mat = align256(p->o_ops + tp.ops.size() * sizeof(TileOp));
        const size_t total = align256(p->o_mat + tp.mats.size() * sizeof(float2));
        check_cuda(cudaStreamSynchronize(e.stream), "plan staging sync");
        char* h = static_cast<char*>(e.host_prog.ensure(total));
        std::memcpy(h + p->o_pass, tp.passes.data(), tp.passes.size() * sizeof(TilePass));
        std::memcpy(h + p->o_phase, tp.phases.data(), tp.phases.size() * sizeof(TilePhase));
        std::memcpy(h + p->o_ops, tp.ops.data(), tp.ops.size() * sizeof(TileOp));
        std::memcpy(h + p->o_mat, tp.mats.data(), tp.mats.size() * sizeof(float2));
        void* d = image ? image->ensure(total) : p->dev.ensure(total);
        p->image = d;
        check_cuda(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, e.stream), "H2D plan");
    } catch (...) {
        delete p;
        throw;
    }
    return p;
}

std::string describe_plan_json(const PlanConfig& cfg, const qlb_gate_instr* prog, uint64_t count,
                               const qlb_pool_view* pool) {
    Planner pl(cfg, pool);
    pl.plan(prog, count);
    std::string out;
    out.reserve(1 << 16);
    auto num = [&](double v) {
        char b[32];
        std::snprintf(b, sizeof b, "%.17g", v);
        out += b;
    };
    auto u = [&](uint64_t v) { out += std::to_string(v); };
    out += "{\"n\":";
    u(cfg.n);
    out += ",\"mode\":";
    u(static_cast<uint64_t>(cfg.mode));
    out += ",\"steps\":[";
    for (size_t i = 0; i < pl.steps.size(); ++i) {
        const PlanStep& st = pl.steps[i];
        if (i) out += ",";
        out += "{\"kind\":";
        u(st.kind);
        out += ",\"index\":";
        u(st.index);
        out += ",\"type\":";
        u(st.instr.type);
        out += ",\"arity\":";
        u(st.instr.flags_arity & 0x0F);
        out += ",\"qubits\":[";
        for (int j = 0; j < 6; ++j) {
            if (j) out += ",";
            u(j < 4 ? st.instr.qubits[j] : st.instr.qubits_ext[j - 4]);
        }
        out += "],\"param\":";
        num(static_cast<double>(st.instr.payload.param));
        out += ",\"mat\":";
        u(st.mat_off);
        out += "}";
    }
    out += "],\"passes\":[";
    for (size_t i = 0; i < pl.prog.passes.size(); ++i) {
        const TilePass& P = pl.prog.passes[i];
        if (i) out += ",";
        out += "{\"tile_pos\":[";
        for (int j = 0; j < kTileQubits; ++j) {
            if (j) out += ",";
            u(P.tile_pos[j]);
        }
        out += "],\"n_low\":";
        u(P.n_low);
        out += ",\"features\":";
        u(P.features);
        out += ",\"post_data\":";
        u(P.post_data);
        out += ",\"post_n\":";
        u(P.post_n);
        out += ",\"phases\":[";
        for (uint32_t ph = P.phase_begin; ph < P.phase_end; ++ph) {
            const TilePhase& T = pl.prog.phases[ph];
            if (ph != P.phase_begin) out += ",";
            out += "{\"reg_pos\":[";
            for (int j = 0; j < kRegQubits; ++j) {
                if (j) out += ",";
                u(T.reg_pos[j]);
            }
            out += "],\"thr_pos\":[";
            for (int j = 0; j < kThreadQubits; ++j) {
                if (j) out += ",";
                u(T.thr_pos[j]);
            }
            out += "],\"flags\":";
            u(T.flags);
            out += ",\"a_thr\":[";
            for (int j = 0; j < kThreadQubits; ++j) {
                if (j) out += ",";
                u(T.a_thr[j]);
            }
            out += "],\"a_reg\":[";
            for (int j = 0; j < kRegQubits; ++j) {
                if (j) out += ",";
                u(T.a_reg[j]);
            }
            out += "],\"ops\":[";
            for (uint32_t o = T.op_begin; o < T.op_end; ++o) {
                const TileOp& op = pl.prog.ops[o];
                if (o != T.op_begin) out += ",";
                out += "{\"kind\":";
                u(op.kind);
                out += ",\"r0\":";
                u(op.r0);
                out += ",\"r1\":";
                u(op.r1);
                out += ",\"k\":";
                u(op.k);
                out += ",\"ctrl_reg\":";
                u(op.ctrl_reg);
                out += ",\"ctrl_mem\":";
                u(op.ctrl_mem);
                out += ",\"flags\":";
                u(op.flags);
                out += ",\"n\":";
                u(op.n);
                out += ",\"code\":";
                u(op.code);
                out += ",\"data\":";
                u(op.data);
                out += ",\"m\":[";
                for (int j = 0; j < 4; ++j) {
                    if (j) out += ",";
                    num(op.m[j].x);
                    out += ",";
                    num(op.m[j].y);
                }
                out += "]";
                if (op.code == OPC_KRON && o + 1 < T.op_end) {   // the five factors, bit 0 first
                    const TileOp& c = pl.prog.ops[o + 1];
                    float q[20];
                    std::memcpy(q, &op.m[0], 32);
                    std::memcpy(q + 8, &c.flags, 16);
                    std::memcpy(q + 12, &c.m[0], 32);
                    out += ",\"kron\":[";
                    for (int j = 0; j < 20; ++j) {
                        if (j) out += ",";
                        num(q[j]);
                    }
                    out += "]";
                }
                out += "}";
            }
            out += "]}";
        }
        out += "]}";
    }
    // the matrix buffer holds float2 matrices and raw words (TC images, sign
    // terms): dump every 32-bit word as an unsigned integer
    out += "],\"mats\":[";
    for (size_t i = 0; i < pl.prog.mats.size(); ++i) {
        uint32_t w[2];
        std::memcpy(w, &pl.prog.mats[i], 8);
        if (i) out += ",";
        u(w[0]);
        out += ",";
        u(w[1]);
    }
    out += "],\"stats\":{\"sweeps\":";
    u(pl.stats.sweeps);
    out += ",\"tile_passes\":";
    u(pl.stats.tile_passes);
    out += ",\"tc_ops\":";
    u(pl.stats.tc_ops);
    out += ",\"chain_passes\":";
    u(pl.stats.chain_passes);
    out += ",\"dense_ops\":";
    u(pl.stats.dense_ops);
    out += ",\"ops\":";
    u(pl.prog.ops.size());
    out += ",\"phases\":";
    u(pl.prog.phases.size());
    out += "}}";
    return out;
}

void run_plan(qlb_engine& e, const qlb_plan& p) {
    if (p.n != e.sv.n) fail(QLB_ERR_INVALID_ARG, "plan was compiled for a different number of qubits");
    if (!e.err_flag.p) {
        e.err_flag.ensure(256);
        check_cuda(cudaMemsetAsync(e.err_flag.p, 0, sizeof(int), e.stream), "clear error flag");
    }
    const char* d = static_cast<const char*>(p.image);
    const float2* mats = reinterpret_cast<const float2*>(d + p.o_mat);
    for (const PlanStep& st : p.steps) {
        switch (st.kind) {
        case STEP_PASS:
            if (st.features & kPassChain) {
                check_cuda(launch_chain_pass(e.sv.d, e.sv.n, reinterpret_cast<const TilePass*>(d + p.o_pass),
                                             reinterpret_cast<const TilePhase*>(d + p.o_phase),
                                             reinterpret_cast<const TileOp*>(d + p.o_ops), mats, st.index,
                                             static_cast<int*>(e.err_flag.p), e.stream),
                           "chain pass");
                break;
            }
            check_cuda(launch_tile_pass(e.sv.d, e.sv.n, reinterpret_cast<const TilePass*>(d + p.o_pass),
                                        reinterpret_cast<const TilePhase*>(d + p.o_phase),
                                        reinterpret_cast<const TileOp*>(d + p.o_ops), mats, st.index,
                                        static_cast<int>(st.features), static_cast<int*>(e.err_flag.p),
                                        e.stream),
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

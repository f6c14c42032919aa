// middle_end.cpp -- the GPU middle end: Middleware::transpile_gpu.
//
// The reference leaves transpile_gpu empty (middleware.hpp:866).  This is its
// B200 counterpart, with the same three passes as transpile_cpu_openmp
// (middleware.hpp:488-524), retargeted:
//   1. DAG::build   -- frontier-linked dependency DAG (middleware.hpp:165-210)
//   2. gate fusion  -- the reference's BFS block growth with its causality
//      check and 2-gate heuristic (middleware.hpp:526-753), generalised:
//      blocks of up to 6 qubits (qubits 4-5 ride in the instruction's pad
//      bytes), RX/RY/RZ/CZ/CP/SWAP/CCX/CSWAP fusable, composition in FP64;
//      with max_fusion_qubits = 4 and the reference fusable set it produces
//      the reference's streams.
//   3. qubit windowing -- chunking + cost-model swaps (middleware.hpp:759-860)
//      with k_safe = the GPU topology's tile window; the safe zone is
//      phys < k_safe (the reference mixes <= and <, :88/:105 vs :801).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <optional>
#include <string>
#include <vector>

#include "engine.h"
#include "tile.h"

namespace qlb {

namespace {

using cd = std::complex<double>;
constexpr uint32_t NUL = 0xFFFFFFFFu;
constexpr int kMaxFuse = 6;

struct Mat {
    uint32_t dim = 0;
    std::vector<cd> a;   // row-major
    Mat() = default;
    explicit Mat(uint32_t d) : dim(d), a(static_cast<size_t>(d) * d, cd(0.0, 0.0)) {}
    cd& operator()(uint32_t r, uint32_t c) { return a[static_cast<size_t>(r) * dim + c]; }
    const cd& operator()(uint32_t r, uint32_t c) const { return a[static_cast<size_t>(r) * dim + c]; }
};

uint32_t arity_of(const qlb_gate_instr& g) { return g.flags_arity & 0x0F; }

struct Node {
    qlb_gate_instr instr;
    uint32_t in[kMaxFuse], out[kMaxFuse];
    bool fused = false;
};

struct Dag {
    std::vector<Node> nodes;
    std::vector<qlb_gate_instr> rewritten;
    // pool: complex128 data + entries
    std::vector<cd> pool;
    std::vector<qlb_matrix_entry> meta;
};

Dag build_dag(const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pv, uint32_t nq) {
    Dag d;
    if (pv && pv->num_matrices) {
        d.pool.assign(reinterpret_cast<const cd*>(pv->data), reinterpret_cast<const cd*>(pv->data) + pv->num_elements);
        d.meta.assign(pv->metadata, pv->metadata + pv->num_matrices);
    }
    d.nodes.reserve(count);
    std::vector<uint32_t> frontier(nq, NUL);
    for (uint64_t i = 0; i < count; ++i) {
        Node n;
        n.instr = prog[i];
        std::fill(n.in, n.in + kMaxFuse, NUL);
        std::fill(n.out, n.out + kMaxFuse, NUL);
        const uint32_t cur = static_cast<uint32_t>(d.nodes.size());
        const uint32_t k = std::min<uint32_t>(arity_of(n.instr), kMaxFuse);
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t q = instr_qubit(n.instr, j);
            if (q >= nq) continue;
            const uint32_t prev = frontier[q];
            n.in[j] = prev;
            if (prev != NUL) {
                Node& p = d.nodes[prev];
                const uint32_t pk = std::min<uint32_t>(arity_of(p.instr), kMaxFuse);
                for (uint32_t t = 0; t < pk; ++t)
                    if (instr_qubit(p.instr, t) == q) {
                        p.out[t] = cur;
                        break;
                    }
            }
            frontier[q] = cur;
        }
        d.nodes.push_back(n);
    }
    return d;
}

// ---- gate matrices (Middleware::get_matrix, middleware.hpp:399-439) --------

bool is_fusable(const qlb_gate_instr& g, bool ref_set) {
    switch (g.type) {
    case QLB_H: case QLB_X: case QLB_Y: case QLB_Z: case QLB_S: case QLB_CX:
    case QLB_UNITARY: case QLB_FUSED_BLOCK:
        return true;
    case QLB_RX: case QLB_RY: case QLB_RZ: case QLB_CZ: case QLB_CP: case QLB_SWAP: case QLB_CCX: case QLB_CSWAP:
        return !ref_set;
    default:
        return false;
    }
}

Mat permutation_matrix(uint32_t k, uint32_t (*f)(uint32_t)) {
    Mat m(1u << k);
    for (uint32_t c = 0; c < m.dim; ++c) m(f(c), c) = 1.0;
    return m;
}

Mat gate_matrix(const qlb_gate_instr& g, const Dag& d) {
    const double r2 = 1.0 / std::sqrt(2.0);
    const double th = static_cast<double>(g.payload.param), h = 0.5 * th;
    const cd I(0.0, 1.0);
    Mat m(2);
    switch (g.type) {
    case QLB_UNITARY: case QLB_FUSED_BLOCK: {
        const qlb_matrix_entry& e = d.meta.at(g.payload.matrix_idx);
        const uint32_t dim = 1u << arity_of(g);
        Mat u(dim);
        std::copy(d.pool.begin() + e.offset, d.pool.begin() + e.offset + e.num_elements, u.a.begin());
        return u;
    }
    case QLB_H: m(0, 0) = r2; m(0, 1) = r2; m(1, 0) = r2; m(1, 1) = -r2; return m;
    case QLB_X: m(0, 1) = 1.0; m(1, 0) = 1.0; return m;
    case QLB_Y: m(0, 1) = -I; m(1, 0) = I; return m;
    case QLB_Z: m(0, 0) = 1.0; m(1, 1) = -1.0; return m;
    case QLB_S: m(0, 0) = 1.0; m(1, 1) = I; return m;
    case QLB_RX: m(0, 0) = std::cos(h); m(0, 1) = -I * std::sin(h); m(1, 0) = -I * std::sin(h); m(1, 1) = std::cos(h); return m;
    case QLB_RY: m(0, 0) = std::cos(h); m(0, 1) = -std::sin(h); m(1, 0) = std::sin(h); m(1, 1) = std::cos(h); return m;
    case QLB_RZ: m(0, 0) = std::polar(1.0, -h); m(1, 1) = std::polar(1.0, h); return m;
    case QLB_CX:   // bit 0 = control (qubits[0]), bit 1 = target
        return permutation_matrix(2, [](uint32_t c) { return (c & 1u) ? (c ^ 2u) : c; });
    case QLB_SWAP:
        return permutation_matrix(2, [](uint32_t c) { return ((c & 1u) << 1) | ((c >> 1) & 1u); });
    case QLB_CCX:  // bits 0,1 = controls, bit 2 = target
        return permutation_matrix(3, [](uint32_t c) { return ((c & 3u) == 3u) ? (c ^ 4u) : c; });
    case QLB_CSWAP: // bit 0 = control, bits 1,2 swapped
        return permutation_matrix(3, [](uint32_t c) {
            return (c & 1u) ? ((c & 1u) | ((c & 2u) << 1) | ((c & 4u) >> 1)) : c;
        });
    case QLB_CZ: case QLB_CP: {
        Mat u(4);
        u(0, 0) = u(1, 1) = u(2, 2) = 1.0;
        u(3, 3) = g.type == QLB_CZ ? cd(-1.0, 0.0) : std::polar(1.0, th);
        return u;
    }
    default: fail(QLB_ERR_INVALID_ARG, "get_matrix: unsupported gate type");
    }
}

// Scatter-expansion of U (bit i <-> sub[i]) to the joint qubits `full`
// (bit j <-> full[j]) (FusionMath::expand_matrix, middleware.hpp:241-312).
Mat expand(const Mat& U, const std::vector<uint32_t>& sub, const std::vector<uint32_t>& full) {
    if (sub == full) return U;           // the same qubits in the same order
    const uint32_t D = 1u << full.size();
    Mat M(D);
    std::vector<uint32_t> pos(sub.size());
    uint32_t submask = 0;
    for (size_t i = 0; i < sub.size(); ++i) {
        pos[i] = static_cast<uint32_t>(std::find(full.begin(), full.end(), sub[i]) - full.begin());
        submask |= 1u << pos[i];
    }
    auto gather = [&](uint32_t x) {
        uint32_t s = 0;
        for (size_t i = 0; i < pos.size(); ++i) s |= ((x >> pos[i]) & 1u) << i;
        return s;
    };
    // M(r, c) = U(gather(r), gather(c)) where r and c agree outside the
    // sub-qubits: for each row, the columns are r's other bits | scat[s]
    const uint32_t K = 1u << sub.size();
    std::vector<uint32_t> scat(K);
    for (uint32_t s = 0; s < K; ++s) {
        uint32_t x = 0;
        for (size_t i = 0; i < pos.size(); ++i) x |= ((s >> i) & 1u) << pos[i];
        scat[s] = x;
    }
    for (uint32_t r = 0; r < D; ++r) {
        const uint32_t rs = gather(r), base = r & ~submask;
        for (uint32_t s = 0; s < K; ++s) M(r, base | scat[s]) = U(rs, s);
    }
    return M;
}

Mat matmul(const Mat& A, const Mat& B) {
    const uint32_t D = A.dim;
    Mat C(D);
    for (uint32_t i = 0; i < D; ++i)
        for (uint32_t k = 0; k < D; ++k) {
            const cd a = A(i, k);
            if (a == cd(0.0, 0.0)) continue;
            for (uint32_t j = 0; j < D; ++j) C(i, j) += a * B(k, j);
        }
    return C;
}

// FusionMath::fuse_matrices (middleware.hpp:315-344): U2 after U1 on the
// sorted union of their qubits.
Mat fuse(const Mat& U1, const std::vector<uint32_t>& q1, const Mat& U2, const std::vector<uint32_t>& q2,
         std::vector<uint32_t>& out_q) {
    out_q = q1;
    for (uint32_t q : q2)
        if (std::find(out_q.begin(), out_q.end(), q) == out_q.end()) out_q.push_back(q);
    std::sort(out_q.begin(), out_q.end());
    if (out_q == q1) {
        // U2 acts inside U1's (sorted) qubits: mix U1's rows within each group
        // of rows that differ only on U2's qubits (no expanded copy of U2)
        const uint32_t D = U1.dim, K = U2.dim;
        uint32_t submask = 0;
        std::vector<uint32_t> scat(K, 0u);
        for (size_t i = 0; i < q2.size(); ++i) {
            const uint32_t p = static_cast<uint32_t>(std::find(q1.begin(), q1.end(), q2[i]) - q1.begin());
            submask |= 1u << p;
            for (uint32_t s = 0; s < K; ++s) scat[s] |= ((s >> i) & 1u) << p;
        }
        Mat M(D);
        for (uint32_t b = 0; b < D; ++b) {
            if (b & submask) continue;
            for (uint32_t s = 0; s < K; ++s) {
                cd* out = &M(b | scat[s], 0);
                for (uint32_t t = 0; t < K; ++t) {
                    const cd u = U2(s, t);
                    if (u == cd(0.0, 0.0)) continue;
                    const cd* in = &U1(b | scat[t], 0);
                    for (uint32_t j = 0; j < D; ++j) out[j] += u * in[j];
                }
            }
        }
        return M;
    }
    return matmul(expand(U2, q2, out_q), expand(U1, q1, out_q));
}

std::vector<uint32_t> qubits_of(const qlb_gate_instr& g) {
    std::vector<uint32_t> q(arity_of(g));
    for (uint32_t j = 0; j < q.size(); ++j) q[j] = instr_qubit(g, j);
    return q;
}

uint32_t store_matrix(Dag& d, const Mat& m, uint32_t k) {
    qlb_matrix_entry e{};
    e.offset = static_cast<uint32_t>(d.pool.size());
    e.num_elements = m.dim * m.dim;
    e.num_qubits = static_cast<uint8_t>(k);
    d.pool.insert(d.pool.end(), m.a.begin(), m.a.end());
    d.meta.push_back(e);
    return static_cast<uint32_t>(d.meta.size() - 1);
}

bool is_dense(const qlb_gate_instr& g) { return g.type == QLB_UNITARY || g.type == QLB_FUSED_BLOCK; }

// pass_gate_fusion (middleware.hpp:526-753), block cap `maxk`.
void pass_gate_fusion(Dag& d, int maxk, bool ref_set) {
    auto& N = d.nodes;
    auto contains = [](const std::vector<uint32_t>& v, uint32_t x) { return std::find(v.begin(), v.end(), x) != v.end(); };
    for (size_t i = 0; i < N.size(); ++i) {
        if (N[i].fused || !is_fusable(N[i].instr, ref_set)) continue;
        if (static_cast<int>(arity_of(N[i].instr)) > maxk) continue;
        std::vector<uint32_t> block{static_cast<uint32_t>(i)};
        std::vector<uint32_t> bq = qubits_of(N[i].instr);
        bool has_dense = is_dense(N[i].instr);
        for (size_t head = 0; head < block.size(); ++head) {
            const uint32_t b = block[head];
            const uint32_t bk = std::min<uint32_t>(arity_of(N[b].instr), kMaxFuse);
            for (uint32_t o = 0; o < bk; ++o) {
                const uint32_t nx = N[b].out[o];
                if (nx == NUL || N[nx].fused || !is_fusable(N[nx].instr, ref_set)) continue;
                if (contains(block, nx)) continue;
                bool causal = true;
                const uint32_t nk = std::min<uint32_t>(arity_of(N[nx].instr), kMaxFuse);
                for (uint32_t t = 0; t < nk && causal; ++t) {
                    const uint32_t p = N[nx].in[t];
                    if (p != NUL && p > i && !contains(block, p)) causal = false;
                }
                if (!causal) continue;
                std::vector<uint32_t> un = bq;
                bool exceeds = false;
                for (uint32_t t = 0; t < nk; ++t) {
                    const uint32_t q = instr_qubit(N[nx].instr, t);
                    if (!contains(un, q)) {
                        if (static_cast<int>(un.size()) >= maxk) {
                            exceeds = true;
                            break;
                        }
                        un.push_back(q);
                    }
                }
                if (exceeds) continue;
                block.push_back(nx);
                bq = un;
                if (is_dense(N[nx].instr)) has_dense = true;
            }
        }
        // heuristic (middleware.hpp:631-634)
        if (block.size() == 1) continue;
        if (block.size() == 2 && !has_dense) continue;

        Mat M = gate_matrix(N[block[0]].instr, d);
        std::vector<uint32_t> cq = qubits_of(N[block[0]].instr);
        for (size_t k = 1; k < block.size(); ++k) {
            std::vector<uint32_t> oq;
            M = fuse(M, cq, gate_matrix(N[block[k]].instr, d), qubits_of(N[block[k]].instr), oq);
            cq = oq;
        }
        const uint32_t csz = static_cast<uint32_t>(cq.size());
        uint32_t bin[kMaxFuse], bout[kMaxFuse];
        for (uint32_t u = 0; u < csz; ++u) {
            const uint32_t q = cq[u];
            uint32_t first_in = NUL, last_out = NUL;
            for (size_t k = 0; k < block.size(); ++k) {
                const Node& nd = N[block[k]];
                bool found = false;
                for (uint32_t j = 0; j < std::min<uint32_t>(arity_of(nd.instr), kMaxFuse); ++j)
                    if (instr_qubit(nd.instr, j) == q) {
                        first_in = nd.in[j];
                        found = true;
                        break;
                    }
                if (found) break;
            }
            for (size_t k = block.size(); k-- > 0;) {
                const Node& nd = N[block[k]];
                bool found = false;
                for (uint32_t j = 0; j < std::min<uint32_t>(arity_of(nd.instr), kMaxFuse); ++j)
                    if (instr_qubit(nd.instr, j) == q) {
                        last_out = nd.out[j];
                        found = true;
                        break;
                    }
                if (found) break;
            }
            bin[u] = first_in;
            bout[u] = last_out;
        }
        const uint32_t midx = store_matrix(d, M, csz);
        Node& A = N[block[0]];
        A.instr.type = QLB_FUSED_BLOCK;
        A.instr.flags_arity = static_cast<uint8_t>((A.instr.flags_arity & 0xF0) | (csz & 0x0F));
        A.instr.payload.matrix_idx = midx;
        A.instr.qubits_ext[0] = A.instr.qubits_ext[1] = 0;
        for (uint32_t u = 0; u < kMaxFuse; ++u) {
            if (u < csz) {
                if (u < 4) A.instr.qubits[u] = static_cast<uint8_t>(cq[u]);
                else A.instr.qubits_ext[u - 4] = static_cast<uint8_t>(cq[u]);
                A.in[u] = bin[u];
                A.out[u] = bout[u];
                if (bin[u] != NUL) {
                    Node& P = N[bin[u]];
                    for (uint32_t j = 0; j < std::min<uint32_t>(arity_of(P.instr), kMaxFuse); ++j)
                        if (contains(block, P.out[j])) P.out[j] = block[0];
                }
                if (bout[u] != NUL) {
                    Node& S = N[bout[u]];
                    for (uint32_t j = 0; j < std::min<uint32_t>(arity_of(S.instr), kMaxFuse); ++j)
                        if (contains(block, S.in[j])) S.in[j] = block[0];
                }
            } else {
                if (u < 4) A.instr.qubits[u] = 255;
                A.in[u] = NUL;
                A.out[u] = NUL;
            }
        }
        for (size_t k = 1; k < block.size(); ++k) N[block[k]].fused = true;
    }
}

// ---- windowing (middleware.hpp:44-132, 759-860) -----------------------------

struct CostModel {
    int type;                 // 0 threshold, 1 greedy, 2 custom
    uint16_t k_safe;
    uint32_t numa_penalty, swap_penalty;
    qlb_cost_model_fn fn;
    void* ctx;

    // ThresholdCostModel::evaluate_swap (:77-118), safe zone phys < k_safe.
    bool evaluate(const std::vector<uint32_t>& freq, const std::vector<uint16_t>& l2p,
                  const std::vector<uint16_t>& p2l, uint16_t& active, uint16_t& victim) const {
        if (type == 2) {
            return fn(ctx, freq.data(), l2p.data(), p2l.data(), static_cast<uint32_t>(freq.size()), &active, &victim) != 0;
        }
        const uint32_t np = type == 1 ? 1u : numa_penalty, sp = type == 1 ? 0u : swap_penalty;
        uint16_t cand = 0xFFFF;
        uint32_t best = 0;
        for (size_t q = 0; q < freq.size(); ++q)
            if (freq[q] > 0 && l2p[q] >= k_safe) {
                const uint32_t ret = freq[q] * np;
                if (ret >= sp && ret > best) {
                    best = ret;
                    cand = static_cast<uint16_t>(q);
                }
            }
        if (cand == 0xFFFF) return false;
        for (size_t v = 0; v < freq.size(); ++v)
            if (l2p[v] < k_safe && freq[v] == 0) {
                active = cand;
                victim = static_cast<uint16_t>(v);
                return true;
            }
        return false;
    }
};

void pass_qubit_windowing(Dag& d, const CostModel& cm, uint32_t nq) {
    std::vector<uint16_t> l2p(nq), p2l(nq);
    for (uint32_t i = 0; i < nq; ++i) l2p[i] = p2l[i] = static_cast<uint16_t>(i);
    d.rewritten.reserve(d.nodes.size());
    std::vector<uint32_t> freq(nq, 0);
    const uint32_t limit = cm.k_safe;
    size_t i = 0;
    while (i < d.nodes.size()) {
        if (d.nodes[i].fused) {
            ++i;
            continue;
        }
        std::fill(freq.begin(), freq.end(), 0u);
        uint32_t uniq = 0;
        size_t j = i;
        while (j < d.nodes.size()) {
            if (d.nodes[j].fused) {
                ++j;
                continue;
            }
            const qlb_gate_instr& g = d.nodes[j].instr;
            uint32_t fresh = 0;
            for (uint32_t t = 0; t < arity_of(g); ++t) {
                const uint32_t q = instr_qubit(g, t);
                if (q < nq && freq[q] == 0) ++fresh;
            }
            if (uniq + fresh > limit && j > i) break;
            for (uint32_t t = 0; t < arity_of(g); ++t) {
                const uint32_t q = instr_qubit(g, t);
                if (q < nq) {
                    if (freq[q] == 0) ++uniq;
                    ++freq[q];
                }
            }
            ++j;
        }
        uint16_t a = 0, v = 0;
        while (cm.evaluate(freq, l2p, p2l, a, v)) {
            if (a >= nq || v >= nq || a == v) fail(QLB_ERR_INVALID_ARG, "cost model proposed an invalid swap");
            const uint16_t pa = l2p[a], pv = l2p[v];
            qlb_gate_instr s{};
            s.type = QLB_GLOBAL_SWAP;
            s.flags_arity = 2;
            std::memset(s.qubits, 255, 4);
            s.qubits[0] = static_cast<uint8_t>(pa);
            s.qubits[1] = static_cast<uint8_t>(pv);
            d.rewritten.push_back(s);
            l2p[a] = pv;
            l2p[v] = pa;
            p2l[pa] = v;
            p2l[pv] = a;
            if (d.rewritten.size() > 64 * (d.nodes.size() + nq)) fail(QLB_ERR_INVALID_ARG, "cost model does not converge");
        }
        for (size_t w = i; w < j; ++w) {
            if (d.nodes[w].fused) continue;
            qlb_gate_instr g = d.nodes[w].instr;
            for (uint32_t t = 0; t < arity_of(g); ++t) {
                const uint32_t q = instr_qubit(g, t);
                if (q < nq) {
                    if (t < 4) g.qubits[t] = static_cast<uint8_t>(l2p[q]);
                    else g.qubits_ext[t - 4] = static_cast<uint8_t>(l2p[q]);
                }
            }
            d.rewritten.push_back(g);
        }
        i = j;
    }
}

}  // namespace
}  // namespace qlb

struct qlb_module {
    std::vector<qlb_gate_instr> program;
    std::vector<std::complex<double>> pool;
    std::vector<qlb_matrix_entry> meta;
};

using namespace qlb;

namespace {
template <typename F>
int guarded_me(F&& f) {
    try {
        f();
        return QLB_OK;
    } catch (const Error& err) {
        set_last_error(err.msg.c_str());
        return err.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return QLB_ERR_OOM;
    } catch (const std::exception& ex) {
        set_last_error(ex.what());
        return QLB_ERR_INVALID_ARG;
    }
}
}  // namespace

extern "C" {

void qlb_transpile_config_default(qlb_transpile_config* c) {
    if (!c) return;
    *c = qlb_transpile_config{};
    c->enable_gate_fusion = 1;        // TranspilerConfig defaults (middleware.hpp:362-386)
    c->enable_hw_awareness = 1;
    c->cost_model_type = 0;
    c->numa_penalty = 10;
    c->swap_penalty = 1;
    c->k_safe = -1;
    c->max_fusion_qubits = 5;
    c->reference_fusable_set = 0;
    c->custom_cost_model = nullptr;
    c->custom_cost_model_ctx = nullptr;
}

// GPUTopology::get_safe_qubit_limit(): the qubits one tile holds on chip.
int qlb_gpu_safe_qubit_limit(uint32_t* out) {
    if (!out) return QLB_ERR_INVALID_ARG;
    *out = static_cast<uint32_t>(kTileQubits);
    return QLB_OK;
}

int qlb_transpile_gpu(const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool, uint32_t nq,
                      const qlb_transpile_config* cfg_in, qlb_module_t* out) {
    return guarded_me([&] {
        if (!out) fail(QLB_ERR_INVALID_ARG, "out is null");
        if (count && !prog) fail(QLB_ERR_INVALID_ARG, "program is null");
        if (nq > 64) fail(QLB_ERR_INVALID_ARG, "too many qubits");
        qlb_transpile_config cfg;
        if (cfg_in) cfg = *cfg_in;
        else qlb_transpile_config_default(&cfg);
        for (uint64_t i = 0; i < count; ++i) {
            const qlb_gate_instr& g = prog[i];
            if (is_dense(g)) {
                const uint32_t k = arity_of(g);
                if (!pool || g.payload.matrix_idx >= pool->num_matrices || k < 1 || k > 6 ||
                    pool->metadata[g.payload.matrix_idx].num_elements != (1u << (2 * k)))
                    fail(QLB_ERR_INVALID_ARG, "dense instruction does not match its UnitaryPool entry");
            }
            for (uint32_t j = 0; j < std::min<uint32_t>(arity_of(g), 6); ++j)
                if (g.type != QLB_BARRIER && instr_qubit(g, j) >= nq) fail(QLB_ERR_INVALID_ARG, "qubit index out of range");
        }
        Dag d = build_dag(prog, count, pool, nq);
        if (cfg.enable_gate_fusion) {
            const int maxk = std::clamp(cfg.max_fusion_qubits, 1, kMaxFuse);
            pass_gate_fusion(d, maxk, cfg.reference_fusable_set != 0);
        }
        if (cfg.enable_hw_awareness) {
            CostModel cm{};
            cm.type = cfg.cost_model_type;
            if (cfg.custom_cost_model) cm.type = 2;
            if (cm.type == 2 && !cfg.custom_cost_model)
                fail(QLB_ERR_INVALID_ARG, "TranspilerConfig: CostModelType::CUSTOM specified but custom_cost_model is null.");
            cm.k_safe = static_cast<uint16_t>(cfg.k_safe >= 0 ? cfg.k_safe : kTileQubits);
            cm.numa_penalty = cfg.numa_penalty;
            cm.swap_penalty = cfg.swap_penalty;
            cm.fn = cfg.custom_cost_model;
            cm.ctx = cfg.custom_cost_model_ctx;
            pass_qubit_windowing(d, cm, nq);
        }
        auto* m = new qlb_module();
        if (!d.rewritten.empty()) {
            m->program = std::move(d.rewritten);
        } else {
            m->program.reserve(d.nodes.size());
            for (const Node& n : d.nodes)
                if (!n.fused) m->program.push_back(n.instr);
        }
        m->pool = std::move(d.pool);
        m->meta = std::move(d.meta);
        *out = m;
    });
}

int qlb_module_destroy(qlb_module_t m) {
    delete m;
    return QLB_OK;
}

int qlb_module_program(qlb_module_t m, const qlb_gate_instr** program, uint64_t* count) {
    if (!m || !program || !count) return QLB_ERR_INVALID_ARG;
    *program = m->program.data();
    *count = m->program.size();
    return QLB_OK;
}

int qlb_module_pool(qlb_module_t m, qlb_pool_view* out) {
    if (!m || !out) return QLB_ERR_INVALID_ARG;
    out->data = reinterpret_cast<const double*>(m->pool.data());
    out->num_elements = m->pool.size();
    out->metadata = m->meta.data();
    out->num_matrices = m->meta.size();
    return QLB_OK;
}

}  // extern "C"

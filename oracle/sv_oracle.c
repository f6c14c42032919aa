/*
 * sv_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, complex128 restatement of the reference simulator's execution
 * engine (Qlassical include/backend/cpu_openmp_engine.hpp) used as the
 * checker for the B200 backend.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the product never does.
 *
 * Deliberate, documented deviations from the reference:
 *   - GLOBAL_SWAP is executed as a real exchange of two physical qubits and
 *     logical order is restored when execute() returns (the reference treats
 *     it as a no-op, cpu_openmp_engine.hpp:217-219, which corrupts windowed
 *     streams).  ORC_FLAG_GLOBAL_SWAP_NOOP reproduces the reference's no-op.
 *   - Two additive diagonal gate types, CZ (0x22) and CP (0x23), which the
 *     reference expresses as 2-qubit UNITARY diagonals.
 *   - UNITARY / FUSED_BLOCK up to 6 qubits (qubits 4,5 in the pad bytes).
 *
 * Parity of this file is pinned against the reference's own known-answer
 * tests (tests/golden) and against the reference engine compiled from its
 * sources (oracle/_ref, see oracle/Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/qlassical_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_FLAG_GLOBAL_SWAP_NOOP 1u

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) {
    cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re };
    return r;
}
static inline cplx cadd(cplx a, cplx b) { cplx r = { a.re + b.re, a.im + b.im }; return r; }

/* ------------------------------------------------------------------ */
/* MT19937-64 (Matsumoto & Nishimura, 2004 published algorithm), the   */
/* generator behind std::mt19937_64 used at cpu_openmp_engine.hpp:252. */
/* ------------------------------------------------------------------ */
typedef struct orc_rng { uint64_t mt[312]; int mti; } orc_rng;

void orc_rng_seed(orc_rng* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->mti = 312;
}

uint64_t orc_rng_next(orc_rng* g) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    if (g->mti >= 312) {
        for (int i = 0; i < 312; ++i) {
            uint64_t x = (g->mt[i] & UM) | (g->mt[(i + 1) % 312] & LM);
            uint64_t xa = x >> 1;
            if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
            g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
        }
        g->mti = 0;
    }
    uint64_t x = g->mt[g->mti++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

/* uniform_real_distribution<double>(0,1) over a 64-bit engine: one draw
 * scaled by 2^-64, clamped below 1 (the canonical-generation rule). */
double orc_rng_uniform(orc_rng* g) {
    double r = (double)orc_rng_next(g) / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* ------------------------------------------------------------------ */
/* Index helpers: state_vector_utils.hpp:23-34                          */
/* ------------------------------------------------------------------ */
static inline uint64_t insert_zero_bit(uint64_t idx, unsigned t) {
    uint64_t mask = (1ULL << t) - 1ULL;
    return (idx & mask) | ((idx & ~mask) << 1);
}

/* Insert zero bits at the ascending positions q[0..k-1]. */
static inline uint64_t insert_zero_bits(uint64_t idx, const unsigned* sorted_q, unsigned k) {
    for (unsigned j = 0; j < k; ++j) idx = insert_zero_bit(idx, sorted_q[j]);
    return idx;
}

/* ------------------------------------------------------------------ */
/* Kernels                                                             */
/* ------------------------------------------------------------------ */

/* Generic 2x2 on target t (single_target_loop, :260-266; apply_h..apply_rz,
 * :337-465 are all instances of this with fixed matrices). */
static void apply_1q(cplx* a, uint64_t dim, unsigned t, const cplx m[4]) {
    int64_t half = (int64_t)(dim / 2);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < half; ++i) {
        uint64_t i0 = insert_zero_bit((uint64_t)i, t), i1 = i0 | (1ULL << t);
        cplx a0 = a[i0], a1 = a[i1];
        a[i0] = cadd(cmul(m[0], a0), cmul(m[1], a1));
        a[i1] = cadd(cmul(m[2], a0), cmul(m[3], a1));
    }
}

/* Gate matrices, built in double from the float parameter exactly as the
 * reference kernels do (cpu_openmp_engine.hpp:408-465; frontend.hpp:93). */
static void gate_matrix_1q(uint8_t type, float param, cplx m[4]) {
    const double r2 = 1.0 / sqrt(2.0);
    double h = (double)param * 0.5, c = cos(h), s = sin(h);
    cplx z = {0, 0}, one = {1, 0};
    switch (type) {
    case QLB_H: m[0] = (cplx){r2, 0}; m[1] = (cplx){r2, 0}; m[2] = (cplx){r2, 0}; m[3] = (cplx){-r2, 0}; break;
    case QLB_X: m[0] = z; m[1] = one; m[2] = one; m[3] = z; break;
    case QLB_Y: m[0] = z; m[1] = (cplx){0, -1}; m[2] = (cplx){0, 1}; m[3] = z; break;
    case QLB_Z: m[0] = one; m[1] = z; m[2] = z; m[3] = (cplx){-1, 0}; break;
    case QLB_S: m[0] = one; m[1] = z; m[2] = z; m[3] = (cplx){0, 1}; break;
    case QLB_RX: m[0] = (cplx){c, 0}; m[1] = (cplx){0, -s}; m[2] = (cplx){0, -s}; m[3] = (cplx){c, 0}; break;
    case QLB_RY: m[0] = (cplx){c, 0}; m[1] = (cplx){-s, 0}; m[2] = (cplx){s, 0}; m[3] = (cplx){c, 0}; break;
    case QLB_RZ: m[0] = (cplx){cos(-h), sin(-h)}; m[1] = z; m[2] = z; m[3] = (cplx){cos(h), sin(h)}; break;
    default: m[0] = one; m[1] = z; m[2] = z; m[3] = one; break;
    }
}

/* Swap a[base|m_a] <-> a[base|m_b] over every base with zero bits at the
 * sorted hole positions (double_hole_loop :270-297 / triple_hole_loop
 * :301-334; apply_cx/swap/ccx/cswap :468-528 are instances). */
static void swap_in_subspace(cplx* a, uint64_t dim, const unsigned* holes, unsigned nh,
                             uint64_t m_a, uint64_t m_b) {
    int64_t iters = (int64_t)(dim >> nh);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < iters; ++i) {
        uint64_t base = insert_zero_bits((uint64_t)i, holes, nh);
        cplx t = a[base | m_a]; a[base | m_a] = a[base | m_b]; a[base | m_b] = t;
    }
}

static void sort_small(unsigned* q, unsigned k) {
    for (unsigned i = 1; i < k; ++i)
        for (unsigned j = i; j > 0 && q[j - 1] > q[j]; --j) { unsigned t = q[j]; q[j] = q[j - 1]; q[j - 1] = t; }
}

/* Phase e^{i phi} on amplitudes with both bits set (CZ: phi = pi). */
static void apply_cphase(cplx* a, uint64_t dim, unsigned q0, unsigned q1, cplx ph) {
    unsigned h[2] = { q0, q1 };
    sort_small(h, 2);
    uint64_t m = (1ULL << q0) | (1ULL << q1);
    int64_t iters = (int64_t)(dim >> 2);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < iters; ++i) {
        uint64_t idx = insert_zero_bits((uint64_t)i, h, 2) | m;
        a[idx] = cmul(a[idx], ph);
    }
}

/* Dense k-qubit unitary, gather -> U*v -> scatter (apply_unitary :539-606):
 * matrix-index bit j <-> qubit q[j] (unsorted), holes at the sorted qubits. */
static void apply_dense(cplx* a, uint64_t dim, const unsigned* q, unsigned k, const cplx* U) {
    unsigned sq[6];
    uint64_t off[64];
    unsigned bs = 1u << k;
    memcpy(sq, q, k * sizeof(unsigned));
    sort_small(sq, k);
    for (unsigned j = 0; j < bs; ++j) {
        uint64_t o = 0;
        for (unsigned b = 0; b < k; ++b) if ((j >> b) & 1u) o |= 1ULL << q[b];
        off[j] = o;
    }
    int64_t iters = (int64_t)(dim >> k);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < iters; ++i) {
        cplx vin[64], vout[64];
        uint64_t base = insert_zero_bits((uint64_t)i, sq, k);
        for (unsigned j = 0; j < bs; ++j) vin[j] = a[base | off[j]];
        for (unsigned r = 0; r < bs; ++r) {
            cplx acc = {0, 0};
            for (unsigned c = 0; c < bs; ++c) acc = cadd(acc, cmul(U[(size_t)r * bs + c], vin[c]));
            vout[r] = acc;
        }
        for (unsigned j = 0; j < bs; ++j) a[base | off[j]] = vout[j];
    }
}

/* Projective measurement (apply_measure :617-671). */
static uint8_t apply_measure(cplx* a, uint64_t dim, unsigned t, orc_rng* g) {
    int64_t half = (int64_t)(dim / 2);
    double p1 = 0.0;
#pragma omp parallel for reduction(+:p1) schedule(static)
    for (int64_t i = 0; i < half; ++i) {
        uint64_t i1 = insert_zero_bit((uint64_t)i, t) | (1ULL << t);
        p1 += a[i1].re * a[i1].re + a[i1].im * a[i1].im;
    }
    double r = orc_rng_uniform(g);
    uint8_t outcome = (r < p1) ? 1 : 0;
    double p = outcome ? p1 : (1.0 - p1);
    if (p < 1e-12) p = 1e-12;
    double inv = 1.0 / sqrt(p);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < half; ++i) {
        uint64_t i0 = insert_zero_bit((uint64_t)i, t), i1 = i0 | (1ULL << t);
        if (outcome) { a[i0].re = a[i0].im = 0.0; a[i1].re *= inv; a[i1].im *= inv; }
        else         { a[i1].re = a[i1].im = 0.0; a[i0].re *= inv; a[i0].im *= inv; }
    }
    return outcome;
}

/* Exchange physical qubits p and v (the intended GLOBAL_SWAP semantics). */
static void swap_qubits(cplx* a, uint64_t dim, unsigned p, unsigned v) {
    if (p == v) return;
    unsigned h[2] = { p, v };
    sort_small(h, 2);
    swap_in_subspace(a, dim, h, 2, 1ULL << p, 1ULL << v);
}

/* ------------------------------------------------------------------ */
/* Dispatch: execute (:143-225)                                         */
/* ------------------------------------------------------------------ */

static unsigned instr_qubit(const qlb_gate_instr* in, unsigned j) {
    return j < 4 ? in->qubits[j] : in->qubits_ext[j - 4];
}

/*
 * Executes `count` instructions on the complex128 state `amps` (2^n complex,
 * interleaved).  Returns 0, or -1 for an unknown instruction (the reference
 * throws runtime_error) / -2 for a bad matrix index.
 */
int orc_execute(double* amps, uint32_t n, const qlb_gate_instr* prog, uint64_t count,
                const qlb_pool_view* pool, orc_rng* rng, uint8_t* meas, uint64_t meas_cap,
                uint64_t* meas_count, unsigned flags) {
    cplx* a = (cplx*)amps;
    uint64_t dim = 1ULL << n;
    unsigned phys_to_log[64];
    int permuted = 0;
    for (unsigned i = 0; i < 64; ++i) phys_to_log[i] = i;

    for (uint64_t g = 0; g < count; ++g) {
        const qlb_gate_instr* in = &prog[g];
        unsigned q0 = in->qubits[0], q1 = in->qubits[1], q2 = in->qubits[2];
        cplx m[4];
        switch (in->type) {
        case QLB_H: case QLB_X: case QLB_Y: case QLB_Z: case QLB_S:
        case QLB_RX: case QLB_RY: case QLB_RZ:
            gate_matrix_1q(in->type, in->payload.param, m);
            apply_1q(a, dim, q0, m);
            break;
        case QLB_CX: {
            unsigned h[2] = { q0, q1 }; sort_small(h, 2);
            swap_in_subspace(a, dim, h, 2, 1ULL << q0, (1ULL << q0) | (1ULL << q1));
            break;
        }
        case QLB_SWAP: {
            unsigned h[2] = { q0, q1 }; sort_small(h, 2);
            swap_in_subspace(a, dim, h, 2, 1ULL << q1, 1ULL << q0);
            break;
        }
        case QLB_CZ: apply_cphase(a, dim, q0, q1, (cplx){-1.0, 0.0}); break;
        case QLB_CP: {
            double phi = (double)in->payload.param;
            apply_cphase(a, dim, q0, q1, (cplx){cos(phi), sin(phi)});
            break;
        }
        case QLB_CCX: {
            unsigned h[3] = { q0, q1, q2 }; sort_small(h, 3);
            uint64_t c = (1ULL << q0) | (1ULL << q1);
            swap_in_subspace(a, dim, h, 3, c, c | (1ULL << q2));
            break;
        }
        case QLB_CSWAP: {
            unsigned h[3] = { q0, q1, q2 }; sort_small(h, 3);
            uint64_t c = 1ULL << q0;
            swap_in_subspace(a, dim, h, 3, c | (1ULL << q2), c | (1ULL << q1));
            break;
        }
        case QLB_UNITARY: case QLB_FUSED_BLOCK: {
            unsigned k = in->flags_arity & 0x0F, q[6];
            if (!pool || in->payload.matrix_idx >= pool->num_matrices || k == 0 || k > 6) return -2;
            const qlb_matrix_entry* e = &pool->metadata[in->payload.matrix_idx];
            if (e->num_elements != (1u << (2 * k))) return -2;
            for (unsigned j = 0; j < k; ++j) q[j] = instr_qubit(in, j);
            apply_dense(a, dim, q, k, (const cplx*)(pool->data + 2 * (uint64_t)e->offset));
            break;
        }
        case QLB_BARRIER: break;
        case QLB_MEASURE: {
            uint8_t o = apply_measure(a, dim, q0, rng);
            if (meas && *meas_count < meas_cap) meas[*meas_count] = o;
            ++*meas_count;
            break;
        }
        case QLB_GLOBAL_SWAP:
            if (!(flags & ORC_FLAG_GLOBAL_SWAP_NOOP)) {
                swap_qubits(a, dim, q0, q1);
                unsigned t = phys_to_log[q0]; phys_to_log[q0] = phys_to_log[q1]; phys_to_log[q1] = t;
                permuted = 1;
            }
            break;
        default:
            return -1;
        }
    }
    /* Restore logical order: move logical qubit L (now at physical p) back to bit L. */
    if (permuted) {
        for (unsigned L = 0; L < n; ++L) {
            unsigned p = L;
            while (phys_to_log[p] != L) ++p;
            if (p != L) {
                swap_qubits(a, dim, p, L);
                unsigned t = phys_to_log[p]; phys_to_log[p] = phys_to_log[L]; phys_to_log[L] = t;
            }
        }
    }
    return 0;
}

/* Convenience: allocate an orc_rng on the heap for ctypes callers. */
orc_rng* orc_rng_create(uint64_t seed) {
    orc_rng* g = (orc_rng*)malloc(sizeof(orc_rng));
    if (g) orc_rng_seed(g, seed);
    return g;
}
void orc_rng_destroy(orc_rng* g) { free(g); }

/* |0...0> initialisation (cpu_state_vector.hpp:54-78). */
void orc_init_zero(double* amps, uint32_t n) {
    uint64_t dim = 1ULL << n;
    memset(amps, 0, dim * 2 * sizeof(double));
    amps[0] = 1.0;
}

/* sum |c|^2 in double (cpu_state_vector.hpp:97-101). */
double orc_norm_sq(const double* amps, uint64_t dim) {
    double s = 0.0;
    int64_t d = (int64_t)dim;
#pragma omp parallel for reduction(+:s) schedule(static)
    for (int64_t i = 0; i < d; ++i) s += amps[2 * i] * amps[2 * i] + amps[2 * i + 1] * amps[2 * i + 1];
    return s;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

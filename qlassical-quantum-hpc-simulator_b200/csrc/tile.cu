// tile.cu -- the persistent register-resident tile kernel (one launch per pass).
//
// One CTA per SM (256 threads, ~220 KB shared memory) walks the pass's tiles.
// Each tile is 2^13 complex64 amplitudes = 2^(13 - n_low) runs of 2^n_low
// contiguous amplitudes.  Two tile buffers hold the tile being computed and
// the next one, whose load (TMA bulk copies for long runs, cp.async for short
// ones, completion counted on an mbarrier) was issued as soon as its buffer
// was free, so HBM reads overlap compute.  A thread holds 32 amplitudes in
// registers; the pass's phases apply their ops as register arithmetic and
// re-split the tile between phases by transposing it through an XOR-swizzled
// buffer (or, for a phase that opens with a tensor-core op, by writing the
// registers straight into that op's operand).  The tile goes back to HBM
// from registers (short runs) or by bulk stores from shared memory.
// HBM traffic: 16 B per amplitude per pass, however many gates the pass holds.
//
// Every mbarrier wait is bounded; on expiry the CTA raises *err, waits (also
// bounded) for its own copy in flight and returns.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_ptx.cuh"
#include "tile.h"

namespace qlb {

namespace {

using namespace ptx;
constexpr uint32_t kTcCols = 256;               // per M-block: D1 (64 columns) | D2 (64 columns)

constexpr int NT = kTileThreads;            // 256
constexpr int NR = 1 << kRegQubits;         // 32
constexpr int TILE = 1 << kTileQubits;      // 8192
// Tiles whose contiguous runs are at least 2^9 amplitudes (4 KB) move by TMA
// bulk copies (at most 16 per tile) in both directions; shorter runs load by
// cp.async and store from registers.
constexpr uint32_t kBulkMinLow = 9;
constexpr size_t kSmemBuffers = 3 * TILE * sizeof(float2);   // 2 TMA buffers + 1 transpose buffer
constexpr size_t kSmemOps = kMaxSmemOps * sizeof(TileOp);
constexpr size_t kSmemPhases = kMaxSmemPhases * sizeof(TilePhase);
constexpr size_t kSmemMisc = 64;             // 2 tile mbarriers, the MMA mbarrier, TMEM address
constexpr size_t kSmemTcB = 16384;           // B operand staging of a tensor-core op
constexpr size_t kSmemTotal = kSmemBuffers + kSmemOps + kSmemPhases + sizeof(TilePass) + kSmemMisc + kSmemTcB;
static_assert((kSmemBuffers + kSmemOps + kSmemPhases + sizeof(TilePass)) % 16 == 0, "mbarriers and B staging alignment");
static_assert(kSmemTotal <= 227 * 1024, "shared memory per CTA");

__device__ __forceinline__ uint32_t fold4(uint32_t i) { return ((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 15u; }

__device__ __forceinline__ uint64_t tile_base(const TilePass& P, uint64_t tile) {
    uint64_t base = 0;
    for (uint32_t j = 0; j < P.n_out; ++j, tile >>= 1)
        if (tile & 1u) base |= uint64_t{1} << P.out_mem[j];
    return base;
}

// Loads one tile into `dst` (linear tile-local layout).  The tile mbarrier
// expects one arrival per thread.  Runs of at least 2^kBulkMinLow amplitudes
// go by TMA bulk copies (one per run, issued by all threads; thread 0 also
// registers the byte count, and the transaction count may dip below zero
// when a copy lands before that, but the phase cannot complete before
// thread 0 arrives).  Shorter runs would need up to 256 bulk copies, which the
// copy engine processes one after another, so they go by 16-byte cp.async
// copies (16 per thread) whose completion each thread's deferred arrival
// reports.
__device__ __forceinline__ void issue_tile_load(float2* dst, const float2* __restrict__ state, const TilePass& P,
                                                uint64_t tile, uint64_t* bar) {
    const uint64_t base = tile_base(P, tile);
    const uint32_t nl = P.n_low;
    if (nl >= kBulkMinLow) {
        const uint32_t chunks = 1u << (kTileQubits - nl);
        const uint32_t bytes = (1u << nl) * static_cast<uint32_t>(sizeof(float2));
        if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, TILE * sizeof(float2));
        for (uint32_t c = threadIdx.x; c < chunks; c += NT) {
            uint64_t g = base;
            for (uint32_t j = nl; j < static_cast<uint32_t>(kTileQubits); ++j)
                if ((c >> (j - nl)) & 1u) g |= uint64_t{1} << P.tile_pos[j];
            bulk_g2s(dst + (static_cast<size_t>(c) << nl), state + g, bytes, bar);
        }
        if (threadIdx.x != 0) mbar_arrive(bar);
        return;
    }
    // Piece i of this thread holds tile-local amplitudes l, l + 1 with
    // l = 512 i + 2 t: bits 1..8 of l come from the thread, bits 9..12 from i
    // (all >= n_low here, so through tile_pos; bits below n_low map to themselves).
    auto mem_bit = [&](uint32_t j) -> uint64_t { return uint64_t{1} << (j < nl ? j : P.tile_pos[j]); };
    uint64_t gt = base;
    for (uint32_t j = 1; j <= 8; ++j)
        if ((threadIdx.x >> (j - 1)) & 1u) gt |= mem_bit(j);
    const uint64_t hb[4] = {mem_bit(9), mem_bit(10), mem_bit(11), mem_bit(12)};
#pragma unroll
    for (uint32_t i = 0; i < 16; ++i) {
        uint64_t g = gt;
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
            if ((i >> k) & 1u) g |= hb[k];
        const uint32_t l = 512u * i + 2u * threadIdx.x;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + l)), "l"(state + g) : "memory");
    }
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// The inverse: the tile, staged in `src` in the same linear layout, goes back
// to HBM by bulk stores (one group per issuing thread).
__device__ __forceinline__ void issue_tile_store(const float2* src, float2* __restrict__ state, const TilePass& P,
                                                 uint64_t tile) {
    const uint64_t base = tile_base(P, tile);
    const uint32_t nl = P.n_low;
    const uint32_t chunks = 1u << (kTileQubits - nl);
    const uint32_t bytes = (1u << nl) * static_cast<uint32_t>(sizeof(float2));
    for (uint32_t c = threadIdx.x; c < chunks; c += NT) {
        uint64_t g = base;
        for (uint32_t j = nl; j < static_cast<uint32_t>(kTileQubits); ++j)
            if ((c >> (j - nl)) & 1u) g |= uint64_t{1} << P.tile_pos[j];
        bulk_s2g(state + g, src + (static_cast<size_t>(c) << nl), bytes);
    }
    bulk_commit();
}

struct PhaseMap {
    uint32_t tp;               // tile-local index bits of the thread
    uint32_t e[kRegQubits];    // tile-local bit of register bit j
    uint32_t st;               // swizzled slot of (thread, register 0)
    uint32_t s[kRegQubits];    // swizzled slot offset of register bit j
    uint64_t gt;               // memory index of (thread, register 0), including the tile base
};

__device__ __forceinline__ PhaseMap make_map(const TilePass& P, const TilePhase& ph, uint64_t base) {
    PhaseMap M;
    uint32_t tp = 0;
    uint64_t g = base;
    const uint32_t t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < kThreadQubits; ++j)
        if ((t >> j) & 1u) {
            tp |= 1u << ph.thr_pos[j];
            g |= uint64_t{1} << P.tile_pos[ph.thr_pos[j]];
        }
    M.tp = tp;
    M.st = tp ^ fold4(tp);
    M.gt = g;
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j) {
        M.e[j] = 1u << ph.reg_pos[j];
        M.s[j] = M.e[j] ^ fold4(M.e[j]);
    }
    return M;
}

__device__ __forceinline__ uint32_t local_of(const PhaseMap& M, int m) {
    uint32_t r = M.tp;
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j)
        if ((m >> j) & 1) r |= M.e[j];
    return r;
}
__device__ __forceinline__ uint32_t slot_of(const PhaseMap& M, int m) {
    uint32_t r = M.st;
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j)
        if ((m >> j) & 1) r ^= M.s[j];
    return r;
}

// ---- register operations ------------------------------------------------

__device__ __forceinline__ void u1_pair(float2& a0, float2& a1, const float2 (&m)[4]) {
    const float2 x = a0, y = a1;
    a0 = cfma(m[1], y, cmul(m[0], x));
    a1 = cfma(m[3], y, cmul(m[2], x));
}
// Real 2x2 with packed f32x2 arithmetic (both components per instruction);
// m_i = (m_i, m_i).
__device__ __forceinline__ void u1r_pair2(float2& a0, float2& a1, float2 m0, float2 m1, float2 m2, float2 m3) {
    const float2 x = a0, y = a1;
    a0 = __ffma2_rn(m1, y, __fmul2_rn(m0, x));
    a1 = __ffma2_rn(m3, y, __fmul2_rn(m2, x));
}
__device__ __forceinline__ void rx_pair(float2& a0, float2& a1, float c, float s) {
    const float2 x = a0, y = a1;
    a0 = make_float2(fmaf(s, y.y, c * x.x), fmaf(-s, y.x, c * x.y));
    a1 = make_float2(fmaf(s, x.y, c * y.x), fmaf(-s, x.x, c * y.y));
}

// Pair loops over register bit R: uncontrolled, and under a register control mask.
template <int R, typename F>
__device__ __forceinline__ void for_pairs(float2 (&v)[NR], F&& f) {
#pragma unroll
    for (int i = 0; i < NR; ++i)
        if (!(i & (1 << R))) f(v[i], v[i | (1 << R)]);
}
template <int R, typename F>
__device__ __forceinline__ void for_pairs_ctl(float2 (&v)[NR], uint32_t cm, F&& f) {
#pragma unroll
    for (int i = 0; i < NR; ++i)
        if (!(i & (1 << R)) && ((static_cast<uint32_t>(i) & cm) == cm)) f(v[i], v[i | (1 << R)]);
}

template <int R0, int R1>
__device__ __forceinline__ void op_swap(float2 (&v)[NR], uint32_t cm) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (!(i & (1 << R0)) || (i & (1 << R1))) continue;   // i: R0 = 1, R1 = 0
        const int j = i ^ (1 << R0) ^ (1 << R1);
        if ((static_cast<uint32_t>(i) & cm) == cm) {
            const float2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
}

template <int R0, int R1>
__device__ __forceinline__ void op_u2(float2 (&v)[NR], const float2* __restrict__ mat, uint32_t cm) {
    float2 M[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) M[i] = __ldg(mat + i);
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & ((1 << R0) | (1 << R1))) continue;
        if ((static_cast<uint32_t>(i) & cm) != cm) continue;
        const int idx[4] = {i, i | (1 << R0), i | (1 << R1), i | (1 << R0) | (1 << R1)};
        float2 in[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) in[c] = v[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float2 acc = cmul(M[r * 4], in[0]);
#pragma unroll
            for (int c = 1; c < 4; ++c) acc = cfma(M[r * 4 + c], in[c], acc);
            v[idx[r]] = acc;
        }
    }
}

template <int K>
__device__ __forceinline__ void op_dense_reg(float2 (&v)[NR], const float2* __restrict__ mat) {
    constexpr int D = 1 << K;
#pragma unroll
    for (int g = 0; g < NR; g += D) {
        float2 out[D];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            const float4* row = reinterpret_cast<const float4*>(mat + r * D);
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < D; c += 2) {
                const float4 w = __ldg(row + c / 2);
                acc = cfma(make_float2(w.x, w.y), v[g + c], acc);
                acc = cfma(make_float2(w.z, w.w), v[g + c + 1], acc);
            }
            out[r] = acc;
        }
#pragma unroll
        for (int r = 0; r < D; ++r) v[g + r] = out[r];
    }
}

// Dense 32 x 32 on all five register bits; the outputs are parked in the
// slots this thread owns in the current layout (`linear` in the first phase,
// swizzled afterwards), which no other thread touches during the phase.
__device__ __forceinline__ void op_dense5(float2 (&v)[NR], const float2* __restrict__ mat, float2* sm,
                                          const PhaseMap& M, bool linear) {
#pragma unroll 1
    for (int r = 0; r < NR; ++r) {
        const float4* row = reinterpret_cast<const float4*>(mat + r * NR);
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < NR; c += 2) {
            const float4 w = __ldg(row + c / 2);
            acc = cfma(make_float2(w.x, w.y), v[c], acc);
            acc = cfma(make_float2(w.z, w.w), v[c + 1], acc);
        }
        uint32_t sl = linear ? M.tp : M.st;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if ((r >> j) & 1) sl = linear ? (sl | M.e[j]) : (sl ^ M.s[j]);
        sm[sl] = acc;
    }
#pragma unroll
    for (int m = 0; m < NR; ++m) v[m] = sm[linear ? local_of(M, m) : slot_of(M, m)];
}

// ---- tensor-core dense op (tcgen05) ----------------------------------------
//
// A 32x32 complex unitary U on the five register qubits, applied to all 256
// register groups of the tile at once:  D = A * B^T with
//   A[row t][k]  = x_t[k],  k = 2 kappa(m) + ri:  Re / Im of amplitude m of thread t
//                  (kappa: a permutation of the 5 register bits, fixed per op)
//   B[n][k]      = real embedding of U, n = 2 r + ro:  B[2r][2c] = Re U_rc,
//                  B[2r][2c+1] = -Im U_rc, B[2r+1][2c] = Im U_rc, B[2r+1][2c+1] = Re U_rc
// (k, n interleave real and imaginary parts) in bf16 split precision:
// D = Ahi*Bhi + Ahi*Blo + Alo*Bhi, FP32 accumulate in tensor memory (rows
// 0..127 -> TMEM columns 0..63, rows 128..255 -> columns 64..127).
// A is K-major with the 128-byte swizzle: row t at byte 128 t, its 16-byte
// chunk j (k = 8j .. 8j+7) at chunk position j ^ (t & 7); 8-row groups 1024 B
// apart (SBO).  B is K-major without swizzle: 8 x 16 B core matrices,
// LBO = 128 B between the K chunks of one row group, SBO = 1024 B between
// 8-row groups.  D column n of row t is read back by thread t.
struct TcCtx {
    uint32_t tmem;        // TMEM base address (lane 0, column base)
    uint64_t* bar;        // MMA-completion mbarrier
    unsigned char* sb;    // 16 KB B staging area
    uint32_t uses;        // completed TC ops of this CTA (parity of the mbarrier)
};

// B (16 KB, L2-resident: every tile of the pass reads the same image) is
// loaded by all threads with plain loads whose latency hides behind the A
// conversion.  Neither a bulk copy (it would queue behind the next tile's
// bulk prefetch in the copy engine) nor cp.async (its wait would include the
// next tile's cp.async prefetch) is independent of the tile pipeline.
constexpr uint32_t kTcBPerThread = kTcBBytes / (16u * NT);
__device__ __forceinline__ void tc_load_b(const float2* __restrict__ bimg, uint4 (&bq)[kTcBPerThread]) {
    const uint4* bsrc = reinterpret_cast<const uint4*>(bimg);
#pragma unroll
    for (uint32_t i = 0; i < kTcBPerThread; ++i) bq[i] = __ldg(bsrc + i * NT + threadIdx.x);
}
// Stores B (the staging area is free: the previous TC op's MMAs have
// completed), makes A and B visible to the tensor core and synchronizes.
__device__ __forceinline__ void tc_store_b_sync(const uint4 (&bq)[kTcBPerThread], TcCtx& tc) {
    uint4* bdst = reinterpret_cast<uint4*>(tc.sb);
#pragma unroll
    for (uint32_t i = 0; i < kTcBPerThread; ++i) bdst[i * NT + threadIdx.x] = bq[i];
    fence_proxy_async();      // generic writes of A and B -> visible to the tensor core
    tc_fence_before();
    __syncthreads();
}
// Thread 0 issues the 16 MMAs of the op (A at a_hi, a_hi + 32 KB): per M-block
// of 128 rows, A_hi x [B_hi | B_lo] as N = 128 into D1 | D2, then A_lo x B_hi
// accumulated into D1; everyone waits for them and reads its row of
// D1 + D2 back into v (this phase's layout).  Returns false if the wait gave
// up (all threads agree).
__device__ __forceinline__ bool tc_mma_readback(float2 (&v)[NR], const unsigned char* a_hi, TcCtx& tc) {
    if (threadIdx.x == 0) {
        tc_fence_after();
        const uint32_t ahi = smem_u32(a_hi), alo = ahi + 32768u, bhi = smem_u32(tc.sb);
#pragma unroll
        for (uint32_t mb = 0; mb < 2; ++mb) {
            const uint32_t d = tc.tmem + mb * 128u;
#pragma unroll
            for (uint32_t s = 0; s < 4; ++s)
                tc_mma(d, umma_desc_a(ahi + mb * 16384u + s * 32u), umma_desc_b(bhi + s * 256u), kTcIdesc128,
                       s > 0 ? 1u : 0u);
#pragma unroll
            for (uint32_t s = 0; s < 4; ++s)
                tc_mma(d, umma_desc_a(alo + mb * 16384u + s * 32u), umma_desc_b(bhi + s * 256u), kTcIdesc64, 1u);
        }
        tc_commit(tc.bar);
    }
    const bool ok = mbar_wait_bounded(tc.bar, tc.uses & 1u);
    ++tc.uses;
    if (__syncthreads_or(!ok)) return false;
    tc_fence_after();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t row = tc.tmem + (((w & 3u) * 32u) << 16) + (w >> 2) * 128u;
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) {
        uint32_t r1[32], r2[32];
        tc_ld_32(row + h * 32u, r1);
        tc_ld_32(row + 64u + h * 32u, r2);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int c = 0; c < 16; ++c)
            v[16 * h + c] = make_float2(__uint_as_float(r1[2 * c]) + __uint_as_float(r2[2 * c]),
                                        __uint_as_float(r1[2 * c + 1]) + __uint_as_float(r2[2 * c + 1]));
    }
    tc_fence_before();
    return true;
}

// Applies one TC op inside a phase (A written from this phase's registers
// into `cur`, kappa = identity); returns false if the MMA wait gave up.
__device__ __forceinline__ bool op_dense_tc(float2 (&v)[NR], const float2* __restrict__ bimg, float2* cur,
                                            TcCtx& tc) {
    unsigned char* a_hi = reinterpret_cast<unsigned char*>(cur);
    uint4 bq[kTcBPerThread];
    tc_load_b(bimg, bq);
    __syncthreads();          // everyone has read `cur`, which now receives A
    tc_write_a(v, a_hi, a_hi + 32768);
    tc_store_b_sync(bq, tc);
    return tc_mma_readback(v, a_hi, tc);
}

// Enters a kPhaseTcEntry phase: the registers of the previous phase go
// straight into the A operand (in `wbuf`, whose previous readers are done) of
// the phase's first op, whose result arrives in the phase's own layout.
__device__ __forceinline__ bool tc_entry(float2 (&v)[NR], const TilePhase& ph, const float2* __restrict__ bimg,
                                         float2* wbuf, TcCtx& tc) {
    unsigned char* a_hi = reinterpret_cast<unsigned char*>(wbuf);
    uint4 bq[kTcBPerThread];
    tc_load_b(bimg, bq);
    uint32_t base = 0;
#pragma unroll
    for (int j = 0; j < kThreadQubits; ++j)
        if ((threadIdx.x >> j) & 1u) base ^= ph.a_thr[j];
    uint32_t d[kRegQubits];
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j) d[j] = ph.a_reg[j];
#pragma unroll
    for (int m = 0; m < NR; ++m) {
        uint32_t off = base;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if ((m >> j) & 1) off ^= d[j];
        uint32_t hi, lo;
        tc_split(v[m], hi, lo);
        *reinterpret_cast<uint32_t*>(a_hi + off) = hi;
        *reinterpret_cast<uint32_t*>(a_hi + 32768u + off) = lo;
    }
    tc_store_b_sync(bq, tc);
    return tc_mma_readback(v, a_hi, tc);
}

// A factor f on the amplitudes whose register index contains mask cm: folded
// into the thread-wide factor (cm = 0) or the factor of one register bit (a
// single bit, the common case: a controlled phase between a register qubit
// and any other), applied later with loops whose structure is fixed at
// compile time; several bits are applied now.
__device__ __forceinline__ void diag_fold(float2 (&v)[NR], float2& T, float2 (&F)[kRegQubits], uint32_t cm,
                                          float2 f) {
    if (cm == 0u) {
        T = cmul(T, f);
    } else if ((cm & (cm - 1u)) == 0u) {
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if (cm == (1u << j)) F[j] = cmul(F[j], f);
    } else {
#pragma unroll
        for (int m = 0; m < NR; ++m)
            if ((static_cast<uint32_t>(m) & cm) == cm) v[m] = cmul(v[m], f);
    }
}

// Copies a DIAG op's data (n_words 16-byte words, at most kDiagStageWords) into the
// B staging area: each thread has two words in flight, so up to 8 KB cost one
// L2 round trip instead of the chain of dependent loads the op's tables and
// term lists would take from global memory.  The area is free:
// a tensor-core op's MMAs have completed when it returns, and a DIAG op that
// staged ends with a barrier.
static_assert(kDiagStageWords * 16u <= kTcBBytes, "DIAG staging fits the B staging area");
__device__ __forceinline__ const float2* diag_stage(const float2* __restrict__ src, uint32_t n_words,
                                                   unsigned char* sb) {
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    uint4* d4 = reinterpret_cast<uint4*>(sb);
    constexpr uint32_t kPer = 2;      // words in flight per thread (registers are scarce here)
#pragma unroll 1
    for (uint32_t b = 0; b < n_words; b += kPer * NT) {
        uint4 t[kPer];
#pragma unroll
        for (uint32_t i = 0; i < kPer; ++i) {
            const uint32_t k = b + i * NT + threadIdx.x;
            if (k < n_words) t[i] = __ldg(s4 + k);
        }
#pragma unroll
        for (uint32_t i = 0; i < kPer; ++i) {
            const uint32_t k = b + i * NT + threadIdx.x;
            if (k < n_words) d4[k] = t[i];
        }
    }
    __syncthreads();
    return reinterpret_cast<const float2*>(sb);
}

// TOP_DIAG: the per-thread factor of the thread/memory-bit terms, the sign
// mask of the mixed pi terms, the per-register-bit factors of the mixed
// terms, then one complex multiply per amplitude and factor.  `tab` is the
// op's data in shared memory (staged by diag_stage) or in global memory:
// plain (generic) loads serve both (a copy of this code per address space
// measured slower: the kernels' code grows).
__device__ __forceinline__ void op_diag(float2 (&v)[NR], const float2* tab, uint32_t flags,
                                        uint32_t n_t, uint32_t n_s, uint32_t n_g, uint64_t gt) {
    const uint32_t has_r = flags & 1u;
    const float2* q = tab + (has_r ? 32 : 0);
    float2 T = make_float2(1.f, 0.f);
    float2 F[kRegQubits];
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j) F[j] = make_float2(1.f, 0.f);
    if (flags & 2u) {
        T = q[threadIdx.x];
        q += 256;
    }
    uint32_t smask = 0;
    if (flags & 4u) {
        smask = reinterpret_cast<const uint32_t*>(q)[threadIdx.x];
        q += 128;
    }
    const uint32_t n_gt = (flags >> 8) & 0xFFu;
    const uint32_t* gcm = reinterpret_cast<const uint32_t*>(q);
    q += 2 * ((n_gt + 3) / 4);
    const float2* gtab = q;
    q += 256 * n_gt;
    const uint4* p = reinterpret_cast<const uint4*>(q);
#pragma unroll 2
    for (uint32_t t = 0; t < n_t; ++t) {
        const uint4 w0 = p[2 * t], w1 = p[2 * t + 1];
        const uint64_t c = (static_cast<uint64_t>(w0.y) << 32) | w0.x;
        const bool on = (gt & c) == c;
        const float2 f = on ? make_float2(__uint_as_float(w0.z), __uint_as_float(w0.w))
                            : make_float2(__uint_as_float(w1.x), __uint_as_float(w1.y));
        T = cmul(T, f);
    }
    p += 2 * n_t;
#pragma unroll 4
    for (uint32_t t = 0; t < n_s; ++t) {
        const uint4 w = p[t];
        const uint64_t c = (static_cast<uint64_t>(w.y) << 32) | w.x;
        smask ^= ((gt & c) == c) ? w.z : 0u;
    }
    p += n_s;
    for (uint32_t g = 0; g < n_gt; ++g) {
        const float2 f = gtab[256 * g + threadIdx.x];
        if (f.x == 1.f && f.y == 0.f) continue;
        diag_fold(v, T, F, gcm[g], f);
    }
    // G groups (one register mask each): the group's factor is a product over
    // its terms (independent loads, unrolled), folded once.
    for (uint32_t g = 0; g < n_g; ++g) {
        const uint4 h = *p;
        ++p;
        float2 gf = make_float2(1.f, 0.f);
#pragma unroll 4
        for (uint32_t k = 0; k < h.y; ++k) {
            const uint4 w = p[k];
            const uint64_t c = (static_cast<uint64_t>(w.y) << 32) | w.x;
            if ((gt & c) == c) gf = cmul(gf, make_float2(__uint_as_float(w.z), __uint_as_float(w.w)));
        }
        p += h.y;
        if (gf.x != 1.f || gf.y != 0.f) diag_fold(v, T, F, h.x, gf);
    }
    if (has_r) {
#pragma unroll
        for (int m = 0; m < NR; ++m) v[m] = cmul(v[m], cmul(T, tab[m]));
    } else if (T.x != 1.f || T.y != 0.f) {
#pragma unroll
        for (int m = 0; m < NR; ++m) v[m] = cmul(v[m], T);
    }
    if (n_gt | n_g) {
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j) {
            if (F[j].x == 1.f && F[j].y == 0.f) continue;
#pragma unroll
            for (int m = 0; m < NR; ++m)
                if ((m >> j) & 1) v[m] = cmul(v[m], F[j]);
        }
    }
    if (smask) {
#pragma unroll
        for (int m = 0; m < NR; ++m) {
            const uint32_t sgn = (smask << (31 - m)) & 0x80000000u;
            v[m].x = __uint_as_float(__float_as_uint(v[m].x) ^ sgn);
            v[m].y = __uint_as_float(__float_as_uint(v[m].y) ^ sgn);
        }
    }
}

__device__ __forceinline__ float2 f2(uint32_t a, uint32_t b) { return make_float2(__uint_as_float(a), __uint_as_float(b)); }

__device__ __forceinline__ void op_cphase(float2 (&v)[NR], uint32_t cm, float2 p) {
#pragma unroll
    for (int i = 0; i < NR; ++i)
        if ((static_cast<uint32_t>(i) & cm) == cm) v[i] = cmul(v[i], p);
}

// One factor of a TOP_KRON op: the real 2x2 q = (m00, m01, m10, m11) on register bit RR.
template <int RR>
__device__ __forceinline__ void kron_bit(float2 (&v)[NR], uint4 q) {
    const float2 m0 = make_float2(__uint_as_float(q.x), __uint_as_float(q.x));
    const float2 m1 = make_float2(__uint_as_float(q.y), __uint_as_float(q.y));
    const float2 m2 = make_float2(__uint_as_float(q.z), __uint_as_float(q.z));
    const float2 m3 = make_float2(__uint_as_float(q.w), __uint_as_float(q.w));
    for_pairs<RR>(v, [&](float2& x, float2& y) { u1r_pair2(x, y, m0, m1, m2, m3); });
}

// Kernel instantiations by code body: 1-qubit, controlled and diagonal ops
// (kLevelNarrow); those plus register SWAPs (kLevelSwaps); uncontrolled
// 1-qubit rotations, diagonal, SWAP, U2 and tensor-core ops (kLevelTc);
// everything, with the FP32 DENSE3-5 handlers (kLevelWide).  A pass runs the smallest that holds its ops: the
// larger bodies cost instruction-fetch stalls.
constexpr int kLevelNarrow = kBodyNarrow, kLevelSwaps = kBodySwaps, kLevelTc = kBodyTc, kLevelWide = kBodyWide;

// The op loop of one phase.  Each op is four 16-byte words; the first holds
// the dispatch code, the register controls and the data offset.
template <int LEVEL>
__device__ __forceinline__ bool run_ops(float2 (&v)[NR], const TilePhase& ph, const TileOp* ops,
                                        const float2* __restrict__ mats, float2* sm, const PhaseMap& M,
                                        bool linear, TcCtx& tc, uint32_t skip = 0) {
    const uint4* rec = reinterpret_cast<const uint4*>(ops);
    for (uint32_t oi = ph.op_begin + skip; oi < ph.op_end; ++oi) {
        const uint4 q0 = rec[4 * oi];
        if (q0.y & 0x00FF0000u) {          // memory controls: a thread-uniform condition
            const uint4 q1 = rec[4 * oi + 1];
            const uint64_t c = (static_cast<uint64_t>(q1.w) << 32) | q1.z;
            if ((M.gt & c) != c) continue;
        }
        const uint32_t cm = q0.z, data = q0.w;
#define QLB_U1R_CASE(RR)                                                                              \
    case OPC_U1R + RR: {                                                                              \
        const uint4 a = rec[4 * oi + 2], b = rec[4 * oi + 3];                                         \
        const float2 m0 = f2(a.x, a.x), m1 = f2(a.z, a.z), m2 = f2(b.x, b.x), m3 = f2(b.z, b.z);      \
        for_pairs<RR>(v, [&](float2& x, float2& y) { u1r_pair2(x, y, m0, m1, m2, m3); });             \
    } break;
#define QLB_RX_CASE(RR)                                                                               \
    case OPC_RX + RR: {                                                                               \
        const uint4 a = rec[4 * oi + 2];                                                              \
        const float c = __uint_as_float(a.x), s = __uint_as_float(a.y);                               \
        for_pairs<RR>(v, [&](float2& x, float2& y) { rx_pair(x, y, c, s); });                         \
    } break;
#define QLB_U1_NC_CASE(RR)                                                                            \
    case OPC_U1 + RR: {                                                                               \
        const uint4 a = rec[4 * oi + 2], b = rec[4 * oi + 3];                                         \
        const float2 m[4] = {f2(a.x, a.y), f2(a.z, a.w), f2(b.x, b.y), f2(b.z, b.w)};                 \
        for_pairs<RR>(v, [&](float2& x, float2& y) { u1_pair(x, y, m); });                            \
    } break;
#define QLB_U1_CASE(RR)                                                                               \
    QLB_U1_NC_CASE(RR)                                                                                \
    case OPC_U1_CTL + RR: {                                                                           \
        const uint4 a = rec[4 * oi + 2], b = rec[4 * oi + 3];                                         \
        const float2 m[4] = {f2(a.x, a.y), f2(a.z, a.w), f2(b.x, b.y), f2(b.z, b.w)};                 \
        for_pairs_ctl<RR>(v, cm, [&](float2& x, float2& y) { u1_pair(x, y, m); });                    \
    } break;
#define QLB_X_CASE(RR)                                                                                \
    case OPC_X + RR:                                                                                  \
        for_pairs<RR>(v, [](float2& x, float2& y) { const float2 t = x; x = y; y = t; });             \
        break;                                                                                        \
    case OPC_X_CTL + RR:                                                                              \
        for_pairs_ctl<RR>(v, cm, [](float2& x, float2& y) { const float2 t = x; x = y; y = t; });     \
        break;
#define QLB_SWAP_CASES                                                                                \
    case OPC_SWAP + reg_pair_index(0, 1): op_swap<0, 1>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(0, 2): op_swap<0, 2>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(0, 3): op_swap<0, 3>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(0, 4): op_swap<0, 4>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(1, 2): op_swap<1, 2>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(1, 3): op_swap<1, 3>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(1, 4): op_swap<1, 4>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(2, 3): op_swap<2, 3>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(2, 4): op_swap<2, 4>(v, cm); break;                                \
    case OPC_SWAP + reg_pair_index(3, 4): op_swap<3, 4>(v, cm); break;
#define QLB_PAIR_CASES(A, B)                                                                          \
    case OPC_SWAP + reg_pair_index(A, B): op_swap<A, B>(v, cm); break;                                \
    case OPC_U2 + reg_pair_index(A, B): op_u2<A, B>(v, mats + data, cm); break;
#define QLB_DIAG_CASE                                                                                 \
    case OPC_DIAG: {                                                                                  \
        const uint32_t n_words = rec[4 * oi + 2].x;    /* 0: read from global memory */              \
        const uint4 q1 = rec[4 * oi + 1];                                                             \
        const bool staged = n_words - 1u < kDiagStageWords;                                           \
        const float2* tab = staged ? diag_stage(mats + data, n_words, tc.sb) : mats + data;           \
        op_diag(v, tab, q1.x, q1.y & 0xFFFFu, q1.y >> 16, cm, M.gt);                                  \
        if (staged) __syncthreads();   /* the staging area is free again */                           \
    } break;
#define QLB_KRON_CASE                                                                                 \
    case OPC_KRON: {                                                                                  \
        kron_bit<0>(v, rec[4 * oi + 2]);                                                              \
        kron_bit<1>(v, rec[4 * oi + 3]);                                                              \
        kron_bit<2>(v, rec[4 * oi + 5]);                                                              \
        kron_bit<3>(v, rec[4 * oi + 6]);                                                              \
        kron_bit<4>(v, rec[4 * oi + 7]);                                                              \
        ++oi;                          /* the continuation record */                                  \
    } break;
#define QLB_COMMON_CASES                                                                              \
    QLB_U1R_CASE(0) QLB_U1R_CASE(1) QLB_U1R_CASE(2) QLB_U1R_CASE(3) QLB_U1R_CASE(4)                   \
    QLB_RX_CASE(0) QLB_RX_CASE(1) QLB_RX_CASE(2) QLB_RX_CASE(3) QLB_RX_CASE(4)                        \
    QLB_U1_CASE(0) QLB_U1_CASE(1) QLB_U1_CASE(2) QLB_U1_CASE(3) QLB_U1_CASE(4)                        \
    QLB_X_CASE(0) QLB_X_CASE(1) QLB_X_CASE(2) QLB_X_CASE(3) QLB_X_CASE(4)                             \
    QLB_DIAG_CASE                                                                                     \
    QLB_KRON_CASE                                                                                     \
    case OPC_CPHASE:                                                                                  \
        op_cphase(v, cm, f2(rec[4 * oi + 2].x, rec[4 * oi + 2].y));                                  \
        break;
        // Multi-qubit ops live only in the wide instantiation, so passes of
        // 1-qubit and diagonal ops run a kernel with a small code body.
        if constexpr (LEVEL == kLevelWide) {
            switch (q0.x & 0xFFFFu) {
                QLB_COMMON_CASES
                QLB_PAIR_CASES(0, 1) QLB_PAIR_CASES(0, 2) QLB_PAIR_CASES(0, 3) QLB_PAIR_CASES(0, 4)
                QLB_PAIR_CASES(1, 2) QLB_PAIR_CASES(1, 3) QLB_PAIR_CASES(1, 4)
                QLB_PAIR_CASES(2, 3) QLB_PAIR_CASES(2, 4) QLB_PAIR_CASES(3, 4)
            case OPC_DENSE3: op_dense_reg<3>(v, mats + data); break;
            case OPC_DENSE4: op_dense_reg<4>(v, mats + data); break;
            case OPC_DENSE5: op_dense5(v, mats + data, sm, M, linear); break;
            case OPC_DENSE_TC:                 // CTA-wide; never controlled
                if (!op_dense_tc(v, mats + data, sm, tc)) return false;
                break;
            default: break;
            }
        } else if constexpr (LEVEL == kLevelTc) {
            // no X, controlled 1-qubit or CPHASE handlers: passes with those run the wide body
            switch (q0.x & 0xFFFFu) {
                QLB_U1R_CASE(0) QLB_U1R_CASE(1) QLB_U1R_CASE(2) QLB_U1R_CASE(3) QLB_U1R_CASE(4)
                QLB_RX_CASE(0) QLB_RX_CASE(1) QLB_RX_CASE(2) QLB_RX_CASE(3) QLB_RX_CASE(4)
                QLB_U1_NC_CASE(0) QLB_U1_NC_CASE(1) QLB_U1_NC_CASE(2) QLB_U1_NC_CASE(3) QLB_U1_NC_CASE(4)
                QLB_DIAG_CASE
                QLB_KRON_CASE
                QLB_PAIR_CASES(0, 1) QLB_PAIR_CASES(0, 2) QLB_PAIR_CASES(0, 3) QLB_PAIR_CASES(0, 4)
                QLB_PAIR_CASES(1, 2) QLB_PAIR_CASES(1, 3) QLB_PAIR_CASES(1, 4)
                QLB_PAIR_CASES(2, 3) QLB_PAIR_CASES(2, 4) QLB_PAIR_CASES(3, 4)
            case OPC_DENSE_TC:                 // CTA-wide; never controlled
                if (!op_dense_tc(v, mats + data, sm, tc)) return false;
                break;
            default: break;
            }
        } else {
            // Runs of uncontrolled rotations of one kind are applied by a
            // loop over a 5-way switch: its merge points are cheaper than
            // the full dispatch's.
            uint32_t code = q0.x & 0xFFFFu;
            if (code - OPC_U1R < 5u || code - OPC_RX < 5u) {
                const uint32_t base = code - OPC_U1R < 5u ? OPC_U1R : OPC_RX;
                for (;;) {
                    if (base == OPC_U1R) {
                        switch (code) {
                            QLB_U1R_CASE(0) QLB_U1R_CASE(1) QLB_U1R_CASE(2) QLB_U1R_CASE(3) QLB_U1R_CASE(4)
                        default: break;
                        }
                    } else {
                        switch (code) {
                            QLB_RX_CASE(0) QLB_RX_CASE(1) QLB_RX_CASE(2) QLB_RX_CASE(3) QLB_RX_CASE(4)
                        default: break;
                        }
                    }
                    if (oi + 1 >= ph.op_end) break;
                    const uint4 nx = rec[4 * (oi + 1)];
                    const uint32_t nc = nx.x & 0xFFFFu;
                    if (nc - base >= 5u || (nx.y & 0x00FF0000u)) break;
                    ++oi;
                    code = nc;
                }
                continue;
            }
            if constexpr (LEVEL == kLevelSwaps) {
                switch (code) {
                    QLB_COMMON_CASES
                    QLB_SWAP_CASES
                default: break;
                }
            } else {
                switch (code) {
                    QLB_COMMON_CASES
                default: break;
                }
            }
        }
    }
    return true;
}
#undef QLB_COMMON_CASES
#undef QLB_KRON_CASE
#undef QLB_U1R_CASE
#undef QLB_RX_CASE
#undef QLB_U1_CASE
#undef QLB_U1_NC_CASE
#undef QLB_DIAG_CASE
#undef QLB_X_CASE
#undef QLB_PAIR_CASES
#undef QLB_SWAP_CASES

// Largest i with work[i].tile_begin <= tile (entries sorted by tile_begin).
__device__ __forceinline__ uint32_t find_work(const TileWork* __restrict__ work, uint32_t n_work, uint64_t tile) {
    uint32_t lo = 0, hi = n_work;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (work[mid].tile_begin <= tile) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One launch applies one pass to each entry of a work list: the launch's
// flattened tile range is the concatenation of the entries' tiles (a single
// state: one entry passed by value, n_work = 0).  A CTA restages the pass
// descriptor, phases and ops in shared memory when its next tile belongs to
// a different pass.
template <int LEVEL>
__global__ void __launch_bounds__(NT, 1)
k_tile_pass(TileWork single, const TileWork* __restrict__ work, uint32_t n_work, const uint32_t* __restrict__ tile_entry,
            uint64_t ntiles, int features, int* __restrict__ err) {
    const int has_tc = features & kPassTensorCores;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2* bufs = reinterpret_cast<float2*>(smem_raw);
    TileOp* sops = reinterpret_cast<TileOp*>(smem_raw + kSmemBuffers);
    TilePhase* sph = reinterpret_cast<TilePhase*>(smem_raw + kSmemBuffers + kSmemOps);
    TilePass* spass = reinterpret_cast<TilePass*>(smem_raw + kSmemBuffers + kSmemOps + kSmemPhases);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + kSmemBuffers + kSmemOps + kSmemPhases + sizeof(TilePass));
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(bar + 4);
    unsigned char* sb = smem_raw + kSmemBuffers + kSmemOps + kSmemPhases + sizeof(TilePass) + kSmemMisc;

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], NT);          // tile loads: one arrival per thread
        mbar_init(&bar[1], NT);
        mbar_init(&bar[2], 1);
        fence_mbar_init();
    }
    if (has_tc && threadIdx.x < 32) {     // warp 0 owns the tensor-memory allocation
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    TcCtx tc{has_tc ? *tmem_holder : 0u, &bar[2], sb, 0u};
    bool failed = false;

    auto entry = [&](uint64_t t) -> TileWork {
        if (!n_work) return single;
        return work[tile_entry ? __ldg(tile_entry + t) : find_work(work, n_work, t)];
    };

    // Stage the entry's pass: its descriptor, phases and (if they fit) ops.
    // Phase op ranges index the program's op array; the shared copy is rebased.
    uint32_t staged = ~0u, nph = 0;
    const TilePass* staged_prog = nullptr;
    const TilePhase* phases = nullptr;
    const TileOp* ops = nullptr;
    const float2* mats = nullptr;
    auto stage = [&](const TileWork& w) {
        const TilePhase* gphases = w.phases;
        const TileOp* gops = w.ops;
        const TilePass& GP = w.passes[w.pass];
        {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(&GP);
            uint32_t* dst = reinterpret_cast<uint32_t*>(spass);
            for (uint32_t i = threadIdx.x; i < sizeof(TilePass) / 4; i += NT) dst[i] = src[i];
        }
        const uint32_t pb = GP.phase_begin, pe = GP.phase_end;
        nph = pe - pb;
        const bool ph_in_smem = nph <= kMaxSmemPhases;
        if (ph_in_smem)
            for (uint32_t i = threadIdx.x; i < nph * sizeof(TilePhase) / 4; i += NT)
                reinterpret_cast<uint32_t*>(sph)[i] = reinterpret_cast<const uint32_t*>(gphases + pb)[i];
        const uint32_t ob = gphases[pb].op_begin, oe = gphases[pe - 1].op_end;
        const bool ops_in_smem = (oe - ob) <= kMaxSmemOps;
        if (ops_in_smem)
            for (uint32_t i = threadIdx.x; i < (oe - ob) * sizeof(TileOp) / 16; i += NT)
                reinterpret_cast<uint4*>(sops)[i] = reinterpret_cast<const uint4*>(gops + ob)[i];
        phases = ph_in_smem ? sph : gphases + pb;
        ops = ops_in_smem ? sops - ob : gops;
        mats = w.mats;
        staged = w.pass;
        staged_prog = w.passes;
    };

    // Pipeline: tile `it` lives in bufs[it & 1] (mbarrier bar[it & 1]).  The
    // load of tile it + 2 is issued as soon as tile it has finished computing
    // (its buffer is then free), so two loads are in flight while a tile is
    // stored and the next one computes.  A finished tile of long runs is
    // staged in the transpose buffer and written back by bulk stores, which
    // drain while the CTA goes on; the next write into that buffer first
    // waits until the stores have read it.
    // The CTA's tiles stride across the grid, over a work list too: tiles of
    // unequal cost (entries of different passes) spread evenly over the CTAs.
    uint64_t tile = blockIdx.x;
    const uint64_t stride = gridDim.x, end = ntiles;
    float2* xbuf = bufs + 2 * static_cast<size_t>(TILE);
    auto issue_load = [&](uint64_t t, uint32_t slot) {
        const TileWork wl = entry(t);
        // the staged shared-memory copy of the pass when it is the same pass
        // (always, for a single state): its address bits are cheap to read
        const bool same = wl.pass == staged && wl.passes == staged_prog;
        issue_tile_load(bufs + static_cast<size_t>(slot) * TILE, wl.state, same ? *spass : wl.passes[wl.pass],
                        t - wl.tile_begin, &bar[slot]);
    };
    if (tile < end) issue_load(tile, 0);
    if (tile + stride < end) issue_load(tile + stride, 1);
    bool store_pending = false;      // uniform: a bulk store may still be reading xbuf
    auto xbuf_free = [&]() {
        if (store_pending) {
            bulk_wait_read();
            __syncthreads();
            store_pending = false;
        }
    };
    uint32_t it = 0;
    for (; tile < end; tile += stride, ++it) {
        const TileWork w = entry(tile);
        if (w.pass != staged || w.passes != staged_prog) {   // uniform: every thread reads the same entry
            __syncthreads();
            stage(w);
            __syncthreads();
        }
        const TilePass& P = *spass;
        const uint32_t b = it & 1u;
        float2* cur = bufs + static_cast<size_t>(b) * TILE;
        const uint64_t next = tile + stride;
        const bool ok = mbar_wait_bounded(&bar[b], (it >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            if (next < end) mbar_wait_bounded(&bar[b ^ 1u], ((it + 1) >> 1) & 1u);
            failed = true;
            break;
        }
        float2* __restrict__ state = w.state;
        const uint64_t base = tile_base(P, tile - w.tile_begin);
        float2 v[NR];
        PhaseMap M = make_map(P, phases[0], base);
#pragma unroll
        for (int m = 0; m < NR; ++m) v[m] = cur[local_of(M, m)];
        bool good = run_ops<LEVEL>(v, phases[0], ops, mats, cur, M, true, tc);
        // Transposes alternate between the transpose buffer and `cur`: the
        // buffer written at transition k was last read at transition k-2,
        // before barrier k-1, so one barrier per transition suffices.
        float2* rbuf = cur;
        for (uint32_t p = 1; p < nph && good; ++p) {
            float2* wbuf = (rbuf == xbuf) ? cur : xbuf;
            if (wbuf == xbuf) xbuf_free();
            if constexpr (LEVEL >= kLevelTc) {
                const TilePhase& ph = phases[p];
                if (ph.flags & kPhaseTcEntry) {
                    const uint32_t data = reinterpret_cast<const uint4*>(ops)[4 * ph.op_begin].w;
                    good = tc_entry(v, ph, mats + data, wbuf, tc);
                    M = make_map(P, ph, base);
                    rbuf = wbuf;
                    if (good) good = run_ops<LEVEL>(v, ph, ops, mats, rbuf, M, false, tc, 1);
                    continue;
                }
            }
#pragma unroll
            for (int m = 0; m < NR; ++m) wbuf[slot_of(M, m)] = v[m];
            __syncthreads();
            M = make_map(P, phases[p], base);
#pragma unroll
            for (int m = 0; m < NR; ++m) v[m] = wbuf[slot_of(M, m)];
            rbuf = wbuf;
            good = run_ops<LEVEL>(v, phases[p], ops, mats, rbuf, M, false, tc);
        }
        if (!good) {     // a tensor-core wait gave up (every thread agrees)
            if (threadIdx.x == 0) atomicExch(err, 2);
            if (next < end) mbar_wait_bounded(&bar[b ^ 1u], ((it + 1) >> 1) & 1u);
            failed = true;
            break;
        }
        if (P.n_low >= kBulkMinLow) {
            // Stage the tile in xbuf (linear layout, as loaded); then cur is free.
            if (store_pending) bulk_wait_read();
            __syncthreads();             // every thread is done with cur and xbuf
#pragma unroll
            for (int m = 0; m < NR; ++m) xbuf[local_of(M, m)] = v[m];
            fence_proxy_async();         // generic accesses of xbuf and cur precede the bulk copies
            __syncthreads();
            issue_tile_store(xbuf, state, P, tile - w.tile_begin);
            store_pending = true;
            if (next + stride < end) issue_load(next + stride, b);
        } else {
            // Short runs: store from registers (the last phase's lanes are
            // tile positions 0..4, so a warp writes runs of >= 64 contiguous bytes).
            __syncthreads();             // every thread is done with cur
            fence_proxy_async();         // ... before the async-proxy writes of the next load
            if (next + stride < end) issue_load(next + stride, b);
            const TilePhase& last = phases[nph - 1];
            uint64_t ge[kRegQubits];
#pragma unroll
            for (int j = 0; j < kRegQubits; ++j) ge[j] = uint64_t{1} << P.tile_pos[last.reg_pos[j]];
#pragma unroll
            for (int m = 0; m < NR; ++m) {
                uint64_t g = M.gt;
#pragma unroll
                for (int j = 0; j < kRegQubits; ++j)
                    if ((m >> j) & 1) g |= ge[j];
                state[g] = v[m];
            }
        }
    }
    bulk_wait_all();                     // this thread's bulk stores are complete
    if (failed && has_tc) mbar_wait_bounded(&bar[2], tc.uses & 1u);   // a late MMA, if any
    tc_fence_before();
    __syncthreads();
    if (has_tc && threadIdx.x < 32) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tc.tmem), "r"(kTcCols) : "memory");
    }
}

// The tile kernel's bounded wait on an mbarrier that nothing completes: it
// must give up after `limit_ns` and report through `err`, leaving the
// context usable.
__global__ void k_wait_selftest(uint64_t limit_ns, int* __restrict__ err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit_ns);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(err, 1);
}

}  // namespace

cudaError_t launch_wait_selftest(uint64_t limit_ns, int* err, cudaStream_t s) {
    k_wait_selftest<<<1, 32, 0, s>>>(limit_ns, err);
    return cudaGetLastError();
}

cudaError_t configure_tile_kernel() {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_tile_pass<kLevelNarrow>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(kSmemTotal));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_pass<kLevelSwaps>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemTotal));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_pass<kLevelTc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemTotal));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_pass<kLevelWide>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemTotal));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    return cudaSuccess;
}

namespace {
void launch_tile_kernel(unsigned grid, const TileWork& single, const TileWork* work, uint32_t n_work,
                        const uint32_t* tile_entry, uint64_t ntiles, int features, int* err, cudaStream_t s) {
    switch (tile_body(features)) {
    case kBodyWide:
        k_tile_pass<kLevelWide><<<grid, NT, kSmemTotal, s>>>(single, work, n_work, tile_entry, ntiles, features, err);
        break;
    case kBodyTc:
        k_tile_pass<kLevelTc><<<grid, NT, kSmemTotal, s>>>(single, work, n_work, tile_entry, ntiles, features, err);
        break;
    case kBodySwaps:
        k_tile_pass<kLevelSwaps><<<grid, NT, kSmemTotal, s>>>(single, work, n_work, tile_entry, ntiles, features, err);
        break;
    default:
        k_tile_pass<kLevelNarrow><<<grid, NT, kSmemTotal, s>>>(single, work, n_work, tile_entry, ntiles, features, err);
        break;
    }
}
}  // namespace

cudaError_t launch_tile_pass(float2* state, uint32_t n, const TilePass* d_passes, const TilePhase* d_phases,
                             const TileOp* d_ops, const float2* d_mats, uint32_t pass_index, int features,
                             int* err, cudaStream_t s) {
    cudaError_t e = configure_tile_kernel();
    if (e != cudaSuccess) return e;
    const uint64_t tiles = uint64_t{1} << (n - kTileQubits);
    uint64_t grid = static_cast<uint64_t>(sm_count());
    if (grid > tiles) grid = tiles;
    const TileWork single{state, 0, d_passes, d_phases, d_ops, d_mats, pass_index, 0};
    launch_tile_kernel(static_cast<unsigned>(grid), single, nullptr, 0, nullptr, tiles, features, err, s);
    return cudaGetLastError();
}

cudaError_t launch_tile_work(const TileWork* d_work, uint32_t n_work, uint64_t total_tiles, int features, int* err,
                             cudaStream_t s, uint32_t max_ctas, const uint32_t* d_tile_entry) {
    if (n_work == 0 || total_tiles == 0) return cudaSuccess;
    cudaError_t e = configure_tile_kernel();
    if (e != cudaSuccess) return e;
    uint64_t grid = static_cast<uint64_t>(sm_count());
    if (max_ctas && grid > max_ctas) grid = max_ctas;
    if (grid > total_tiles) grid = total_tiles;
    const TileWork none{nullptr, 0, nullptr, nullptr, nullptr, nullptr, 0, 0};
    launch_tile_kernel(static_cast<unsigned>(grid), none, d_work, n_work, d_tile_entry, total_tiles, features, err, s);
    return cudaGetLastError();
}

}  // namespace qlb

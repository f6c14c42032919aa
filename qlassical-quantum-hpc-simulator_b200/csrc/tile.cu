// tile.cu -- the register-resident tile kernel (one launch per pass).
//
// Each CTA (256 threads) owns one tile of 2^13 complex64 amplitudes: the
// amplitudes whose non-tile index bits equal the CTA's tile number.  A
// thread holds 32 amplitudes in registers (5 "register qubits"), the
// thread index covers the other 8 tile qubits.  The pass is a list of
// phases; each phase applies its instructions purely in registers, and
// consecutive phases re-split the tile qubits by transposing the tile
// through 64 KB of XOR-swizzled shared memory.  The first phase reads the
// tile straight from HBM and the last phase writes it straight back; both
// use lanes = memory qubits 0..4, so every warp request is 256 contiguous
// bytes.  HBM traffic: 16 B per amplitude per pass, independent of how many
// instructions the pass absorbs.
#include "common.cuh"
#include "tile.h"

namespace qlb {

namespace {

constexpr int NT = kTileThreads;            // 256
constexpr int NR = 1 << kRegQubits;         // 32
constexpr int TILE = 1 << kTileQubits;      // 8192

__device__ __forceinline__ uint32_t fold4(uint32_t i) { return ((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 15u; }

struct PhaseMap {
    uint32_t st;          // swizzled shared-memory slot of the thread's register 0
    uint32_t s[kRegQubits];  // slot offset (XOR) of register bit j
    uint64_t gt;          // memory index of the thread's register 0
    uint64_t ge[kRegQubits]; // memory bit of register bit j
};

__device__ __forceinline__ PhaseMap make_map(const TilePass& P, const TilePhase& ph, uint64_t base) {
    PhaseMap M;
    uint32_t tpart = 0;
    uint64_t gmem = base;
    const uint32_t t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < kThreadQubits; ++j) {
        if ((t >> j) & 1u) {
            tpart |= 1u << ph.thr_pos[j];
            gmem |= uint64_t{1} << P.tile_pos[ph.thr_pos[j]];
        }
    }
    M.st = tpart ^ fold4(tpart);
    M.gt = gmem;
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j) {
        const uint32_t e = 1u << ph.reg_pos[j];
        M.s[j] = e ^ fold4(e);
        M.ge[j] = uint64_t{1} << P.tile_pos[ph.reg_pos[j]];
    }
    return M;
}

__device__ __forceinline__ uint32_t slot_of(const PhaseMap& M, int m) {
    uint32_t r = M.st;
    if (m & 1) r ^= M.s[0];
    if (m & 2) r ^= M.s[1];
    if (m & 4) r ^= M.s[2];
    if (m & 8) r ^= M.s[3];
    if (m & 16) r ^= M.s[4];
    return r;
}

__device__ __forceinline__ uint64_t gaddr(const PhaseMap& M, int m) {
    uint64_t r = M.gt;
    if (m & 1) r |= M.ge[0];
    if (m & 2) r |= M.ge[1];
    if (m & 4) r |= M.ge[2];
    if (m & 8) r |= M.ge[3];
    if (m & 16) r |= M.ge[4];
    return r;
}

// ---- register operations ------------------------------------------------

template <int R>
__device__ __forceinline__ void op_u1(float2 (&v)[NR], const float2 (&m)[4], uint32_t cm) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << R)) continue;
        const int j = i | (1 << R);
        if ((static_cast<uint32_t>(i) & cm) == cm) {
            const float2 a0 = v[i], a1 = v[j];
            v[i] = cfma(m[1], a1, cmul(m[0], a0));
            v[j] = cfma(m[3], a1, cmul(m[2], a0));
        }
    }
}

template <int R>
__device__ __forceinline__ void op_x(float2 (&v)[NR], uint32_t cm) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
        if (i & (1 << R)) continue;
        const int j = i | (1 << R);
        if ((static_cast<uint32_t>(i) & cm) == cm) {
            const float2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
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
        float2 in[4], out[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) in[c] = v[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float2 acc = cmul(M[r * 4], in[0]);
#pragma unroll
            for (int c = 1; c < 4; ++c) acc = cfma(M[r * 4 + c], in[c], acc);
            out[r] = acc;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) v[idx[r]] = out[r];
    }
}

// Dense 2^K x 2^K on register bits 0..K-1 (K = 3, 4): groups of 2^K
// consecutive registers.
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

// Dense 32 x 32 on all five register bits; outputs are parked in the
// thread's own shared-memory slots (no other thread touches them during a
// phase) to keep register pressure bounded.
__device__ __forceinline__ void op_dense5(float2 (&v)[NR], const float2* __restrict__ mat, float2* sm,
                                          const PhaseMap& M) {
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
        uint32_t sl = M.st;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if ((r >> j) & 1) sl ^= M.s[j];
        sm[sl] = acc;
    }
#pragma unroll
    for (int m = 0; m < NR; ++m) {
        uint32_t sl = M.st;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if ((m >> j) & 1) sl ^= M.s[j];
        v[m] = sm[sl];
    }
}

// Phase polynomial.  Layout of pdata (uint32) at op.data:
//   [0] constant angle, [1..5] unconditional h_j, [6..15] q_{jk} (j<k,
//   lexicographic), [16] number of thread terms T, [17] number of linear
//   conditional terms L, then T words (ga | gb << 8) + T angles, then
//   L words (j | gb << 8) + L angles.  Angles are turns * 2^32.
__device__ __forceinline__ void op_phase(float2 (&v)[NR], const uint32_t* __restrict__ pd, uint64_t gt) {
    uint32_t acc = __ldg(pd + 0);
    uint32_t h[kRegQubits], q[10];
#pragma unroll
    for (int j = 0; j < kRegQubits; ++j) h[j] = __ldg(pd + 1 + j);
#pragma unroll
    for (int j = 0; j < 10; ++j) q[j] = __ldg(pd + 6 + j);
    const uint32_t T = __ldg(pd + 16), L = __ldg(pd + 17);
    const uint32_t* tw = pd + 18;
    for (uint32_t i = 0; i < T; ++i) {
        const uint32_t w = __ldg(tw + 2 * i), ang = __ldg(tw + 2 * i + 1);
        const uint32_t ga = w & 0xFFu, gb = (w >> 8) & 0xFFu;
        const bool on = ((gt >> ga) & 1u) && (gb == 0xFFu || ((gt >> gb) & 1u));
        acc += on ? ang : 0u;
    }
    const uint32_t* lw = tw + 2 * T;
    for (uint32_t i = 0; i < L; ++i) {
        const uint32_t w = __ldg(lw + 2 * i), ang = __ldg(lw + 2 * i + 1);
        const uint32_t j = w & 0xFFu, gb = (w >> 8) & 0xFFu;
        const uint32_t add = (gb == 0xFFu || ((gt >> gb) & 1u)) ? ang : 0u;
#pragma unroll
        for (int jj = 0; jj < kRegQubits; ++jj) h[jj] += (j == static_cast<uint32_t>(jj)) ? add : 0u;
    }
    constexpr float kTurnToRad = 6.283185307179586f / 4294967296.0f;
#pragma unroll
    for (int m = 0; m < NR; ++m) {
        uint32_t phi = acc;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
            if ((m >> j) & 1) phi += h[j];
        int pi = 0;
#pragma unroll
        for (int j = 0; j < kRegQubits; ++j)
#pragma unroll
            for (int k = j + 1; k < kRegQubits; ++k) {
                if (((m >> j) & 1) && ((m >> k) & 1)) phi += q[pi];
                ++pi;
            }
        if (phi != 0u) {
            float sn, cs;
            __sincosf(static_cast<float>(static_cast<int32_t>(phi)) * kTurnToRad, &sn, &cs);
            v[m] = cmul(v[m], make_float2(cs, sn));
        }
    }
}

#define QLB_R1(r, STMT)                      \
    switch (r) {                             \
    case 0: { constexpr int R = 0; STMT; } break; \
    case 1: { constexpr int R = 1; STMT; } break; \
    case 2: { constexpr int R = 2; STMT; } break; \
    case 3: { constexpr int R = 3; STMT; } break; \
    default: { constexpr int R = 4; STMT; } break; \
    }

#define QLB_R2(a, b, STMT)                                              \
    switch ((a) * 8 + (b)) {                                            \
    case 0 * 8 + 1: { constexpr int A = 0, B = 1; STMT; } break;        \
    case 0 * 8 + 2: { constexpr int A = 0, B = 2; STMT; } break;        \
    case 0 * 8 + 3: { constexpr int A = 0, B = 3; STMT; } break;        \
    case 0 * 8 + 4: { constexpr int A = 0, B = 4; STMT; } break;        \
    case 1 * 8 + 2: { constexpr int A = 1, B = 2; STMT; } break;        \
    case 1 * 8 + 3: { constexpr int A = 1, B = 3; STMT; } break;        \
    case 1 * 8 + 4: { constexpr int A = 1, B = 4; STMT; } break;        \
    case 2 * 8 + 3: { constexpr int A = 2, B = 3; STMT; } break;        \
    case 2 * 8 + 4: { constexpr int A = 2, B = 4; STMT; } break;        \
    default: { constexpr int A = 3, B = 4; STMT; } break;               \
    }

__device__ __forceinline__ void run_ops(float2 (&v)[NR], const TilePhase& ph, const TileOp* __restrict__ ops,
                                        const uint32_t* __restrict__ pdata, const float2* __restrict__ mats,
                                        float2* sm, const PhaseMap& M) {
    for (uint32_t oi = ph.op_begin; oi < ph.op_end; ++oi) {
        const TileOp& op = ops[oi];
        const uint8_t kind = op.kind;
        if (kind == TOP_PHASE) {
            op_phase(v, pdata + op.data, M.gt);
            continue;
        }
        if ((M.gt & op.ctrl_mem) != op.ctrl_mem) continue;   // thread-uniform control
        const uint32_t cm = op.ctrl_reg;
        switch (kind) {
        case TOP_U1: {
            float2 m[4] = {op.m[0], op.m[1], op.m[2], op.m[3]};
            QLB_R1(op.r0, op_u1<R>(v, m, cm));
            break;
        }
        case TOP_X: QLB_R1(op.r0, op_x<R>(v, cm)); break;
        case TOP_SWAP: QLB_R2(op.r0, op.r1, (op_swap<A, B>(v, cm))); break;
        case TOP_U2: QLB_R2(op.r0, op.r1, (op_u2<A, B>(v, mats + op.data, cm))); break;
        case TOP_DENSE:
            if (op.k == 3) op_dense_reg<3>(v, mats + op.data);
            else if (op.k == 4) op_dense_reg<4>(v, mats + op.data);
            else op_dense5(v, mats + op.data, sm, M);
            break;
        default: break;
        }
    }
}

__global__ void __launch_bounds__(NT, 1)
k_tile_pass(float2* __restrict__ state, const TilePass* __restrict__ passes, const TilePhase* __restrict__ phases,
            const TileOp* __restrict__ ops, const uint32_t* __restrict__ pdata, const float2* __restrict__ mats,
            uint32_t pass_index) {
    extern __shared__ float2 sm[];
    const TilePass& P = passes[pass_index];

    // tile base: deposit the CTA index into the non-tile memory qubits
    uint64_t base = 0;
    {
        uint64_t b = blockIdx.x;
        for (uint32_t j = 0; j < P.n_out; ++j, b >>= 1)
            if (b & 1u) base |= uint64_t{1} << P.out_mem[j];
    }

    float2 v[NR];
    const uint32_t pb = P.phase_begin, pe = P.phase_end;
    PhaseMap M = make_map(P, phases[pb], base);
#pragma unroll
    for (int m = 0; m < NR; ++m) v[m] = state[gaddr(M, m)];
    run_ops(v, phases[pb], ops, pdata, mats, sm, M);

    for (uint32_t p = pb + 1; p < pe; ++p) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < NR; ++m) sm[slot_of(M, m)] = v[m];
        __syncthreads();
        M = make_map(P, phases[p], base);
#pragma unroll
        for (int m = 0; m < NR; ++m) v[m] = sm[slot_of(M, m)];
        run_ops(v, phases[p], ops, pdata, mats, sm, M);
    }
#pragma unroll
    for (int m = 0; m < NR; ++m) state[gaddr(M, m)] = v[m];
}

}  // namespace

cudaError_t launch_tile_pass(float2* state, uint32_t n, const TilePass* d_pass, const TilePhase* d_phases,
                             const TileOp* d_ops, const uint32_t* d_pdata, const float2* d_mats,
                             uint32_t pass_index, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_tile_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             TILE * static_cast<int>(sizeof(float2)));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const uint64_t tiles = uint64_t{1} << (n - kTileQubits);
    k_tile_pass<<<static_cast<unsigned>(tiles), NT, TILE * sizeof(float2), s>>>(
        state, d_pass, d_phases, d_ops, d_pdata, d_mats, pass_index);
    return cudaGetLastError();
}

}  // namespace qlb

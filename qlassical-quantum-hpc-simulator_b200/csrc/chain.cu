// chain.cu -- the tensor-core chain kernel: one launch per chain pass.
//
// A chain pass is a tile pass whose register phases each hold one op, a
// 32 x 32 complex unitary on the phase's five register qubits applied by
// tcgen05 split-bf16 MMAs (A = the tile, 256 rows; B = the unitary's real
// embedding, hi/lo; FP32 accumulate in tensor memory; the operand layouts
// are the general tile kernel's, tile.cu).  Between two ops the tile never
// visits the register file longer than one conversion: tensor memory ->
// registers (D1 + D2) -> bf16 hi/lo -> the next op's A operand in shared
// memory, scattered by the planner's per-bit XOR offsets.
//
// Where the general kernel runs one tile at a time and waits for every
// MMA, this one keeps two tiles in flight per SM ("slots", each with 256
// tensor-memory columns and its own B staging): while slot 0's MMAs run,
// the 256 compute threads convert slot 1's tile, and the other way round.
// Slot 1 starts half a tile behind slot 0, so its buffer's next load has
// time to land.  One thread of a ninth warp moves every tile between HBM and
// three 64 KB buffers with TMA tensor copies: the state is viewed as a
// 5-dimensional tensor whose dimensions start at the tile's runs of
// consecutive memory qubits, so a tile is one box (or a few, when it has
// more than five runs) and a copy's coordinates are the tile's other
// qubits.  The last op's result is staged in its buffer in tile order and
// stored by the same thread, which then reloads the buffer.  A tenth warp
// issues the MMAs: a slot's 256 threads arrive on its "A ready" barrier
// after writing A and B and go on to the other slot at once, so an MMA
// issue that waits for the tensor pipe to drain the other slot's MMAs
// stalls nobody.  HBM traffic: 16 B per amplitude per pass.
//
// Every wait is bounded (2 s / 2^26 polls); on expiry the CTA raises *err,
// waits (bounded) for its own MMAs and copies, frees its tensor memory and
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "tc_ptx.cuh"
#include "tile.h"

namespace qlb {

namespace {

using namespace ptx;

constexpr int kCompute = 256;                     // thread t converts A / D row t
constexpr int kLoadWarp = kCompute;               // first thread of the load warp
constexpr int kMmaWarp = kCompute + 32;           // first thread of the MMA warp
constexpr int kThreads = kCompute + 64;
constexpr uint32_t kTile = 1u << kTileQubits;
constexpr uint32_t kBufBytes = kTile * 8u;        // 64 KB: the tile (fp32) or its A operand (bf16 hi | lo)
constexpr uint32_t kBufs = 3;
constexpr size_t kOffB = size_t{kBufs} * kBufBytes;
constexpr size_t kOffPass = kOffB + 2 * kTcBBytes;
constexpr size_t kOffPhases = kOffPass + sizeof(TilePass);
constexpr size_t kOffBoff = kOffPhases + kMaxSmemPhases * sizeof(TilePhase);
constexpr size_t kOffBar = (kOffBoff + kMaxSmemPhases * 4 + 7) & ~size_t{7};
// mbarriers: full[3], staged[3], mma[2], aready[2]; then the tensor-memory
// address and the two slots' MMA mailboxes (A, B, D addresses)
constexpr size_t kSmemChain = kOffBar + 10 * 8 + 8 + 2 * 16;
static_assert(sizeof(TilePass) % 8 == 0 && sizeof(TilePhase) % 4 == 0, "descriptor staging");
static_assert(kSmemChain <= 227 * 1024, "shared memory per CTA");
constexpr uint32_t kBPerThread = kTcBBytes / (16u * kCompute);   // 4 x 16 B of B per thread
constexpr uint32_t kTmemCols = 512;               // two slots x (2 M-blocks x (D1 | D2))

// The tile as TMA boxes: the state is a 5-D tensor of 8-byte amplitudes
// whose dimension d covers memory qubits [lo[d], lo[d+1]) (the last real
// one up to n); a tile's runs of consecutive memory qubits (at most 8 per
// dimension) sit at the bottom of the first five dimensions, so a box holds
// them in tile order.  Tile qubits beyond the fifth run (rem_q, ascending)
// are enumerated by 2^n_rem copies of box_bytes each, in tile order too.
// A tile's coordinates are its out qubits, each at bit (q - lo[d]) of the
// dimension d that contains it.
struct ChainGeom {
    uint8_t lo[5];       // first memory qubit of each dimension (64: unused dimension)
    uint8_t n_rem;
    uint8_t rem_q[13];
    uint8_t pad[3];
    uint32_t box_bytes;
};

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, const int (&c)[5], uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, const int (&c)[5], uint32_t src) {
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(src)
                 : "memory");
}

// Coordinates of copy `cpy` of tile `tile`.
__device__ __forceinline__ void tile_coords(const TilePass& P, const ChainGeom& g, uint64_t tile, uint32_t cpy,
                                            int (&c)[5]) {
#pragma unroll
    for (int d = 0; d < 5; ++d) c[d] = 0;
    for (uint32_t j = 0; j < P.n_out; ++j, tile >>= 1) {
        if (!(tile & 1u)) continue;
        const uint32_t q = P.out_mem[j];
        int d = 0;
#pragma unroll
        for (int k = 1; k < 5; ++k)
            if (g.lo[k] <= q) d = k;
        c[d] |= 1 << (q - g.lo[d]);
    }
    for (uint32_t i = 0; i < g.n_rem; ++i)
        if ((cpy >> i) & 1u) c[4] |= 1 << (g.rem_q[i] - g.lo[4]);
}

// Barrier 1 over the 256 compute threads (the load warp never joins it).
__device__ __forceinline__ void compute_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
__device__ __forceinline__ bool compute_any(bool x) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 256, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(x ? 1u : 0u)
        : "memory");
    return r != 0;
}

// Issues the 16 MMAs of one op on A at `a` (hi; lo 32 KB above), B at `b`,
// D at tensor-memory column `d`: per M-block of 128 rows, A_hi x [B_hi |
// B_lo] (N = 128) into D1 | D2, then A_lo x B_hi (N = 64) added into D1.
__device__ __forceinline__ void issue_mmas(uint32_t a, uint32_t b, uint32_t d, uint64_t* bar) {
    tc_fence_after();   // after the wait that saw A and B written (and the previous D read)
#pragma unroll
    for (uint32_t mb = 0; mb < 2; ++mb) {
        const uint32_t dm = d + mb * 128u;
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s)
            tc_mma(dm, umma_desc_a(a + mb * 16384u + s * 32u), umma_desc_b(b + s * 256u), kTcIdesc128, s > 0 ? 1u : 0u);
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s)
            tc_mma(dm, umma_desc_a(a + 32768u + mb * 16384u + s * 32u), umma_desc_b(b + s * 256u), kTcIdesc64, 1u);
    }
    tc_commit(bar);
}

// Reads 16 amplitudes (register indices 16 h .. 16 h + 15) of this thread's
// D row: D1 + D2, columns 32 h .. 32 h + 31 of each.
__device__ __forceinline__ void read_half(uint32_t row, uint32_t h, float2 (&a)[16]) {
    uint32_t r1[32], r2[32];
    tc_ld_32(row + h * 32u, r1);
    tc_ld_32(row + 64u + h * 32u, r2);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 16; ++c)
        a[c] = make_float2(__uint_as_float(r1[2 * c]) + __uint_as_float(r2[2 * c]),
                           __uint_as_float(r1[2 * c + 1]) + __uint_as_float(r2[2 * c + 1]));
}

// Scatters amplitudes with register indices base_r .. base_r + 15 into the
// A operand at `a` (hi; lo 32 KB above): byte offset = thread part ^ XOR of
// d[i] over the index's set bits.
__device__ __forceinline__ void scatter16(const float2 (&v)[16], uint32_t base_r, uint32_t thr_off,
                                          const uint32_t (&d)[kRegQubits], unsigned char* a) {
#pragma unroll
    for (uint32_t c = 0; c < 16; ++c) {
        const uint32_t r = base_r + c;
        uint32_t off = thr_off;
#pragma unroll
        for (int i = 0; i < kRegQubits; ++i)
            if ((r >> i) & 1u) off ^= d[i];
        uint32_t hi, lo;
        tc_split(v[c], hi, lo);
        *reinterpret_cast<uint32_t*>(a + off) = hi;
        *reinterpret_cast<uint32_t*>(a + 32768u + off) = lo;
    }
}

__global__ void __launch_bounds__(kThreads, 1)
k_tc_chain(const __grid_constant__ CUtensorMap tmap, const ChainGeom geom, TileWork w, uint64_t ntiles,
           int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* bufs = smem;
    unsigned char* bstage = smem + kOffB;
    TilePass* sp = reinterpret_cast<TilePass*>(smem + kOffPass);
    TilePhase* sph = reinterpret_cast<TilePhase*>(smem + kOffPhases);
    uint32_t* sboff = reinterpret_cast<uint32_t*>(smem + kOffBoff);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kOffBar);    // [3] tile loaded
    uint64_t* staged = full + 3;                                     // [3] a tile's result staged
    uint64_t* mmab = full + 6;                                       // [2] a slot's MMAs done
    uint64_t* aready = full + 8;                                     // [2] a slot's A and B written
    uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(full + 10);
    uint32_t* mbox = tmem_holder + 2;                                // [2][4] A, B, D of a slot's next op
    const uint32_t tid = threadIdx.x;

    // ---- set-up: the pass descriptor, its phases, the ops' B offsets ----
    {
        const TilePass& GP = w.passes[w.pass];
        for (uint32_t i = tid; i < sizeof(TilePass) / 4; i += kThreads)
            reinterpret_cast<uint32_t*>(sp)[i] = reinterpret_cast<const uint32_t*>(&GP)[i];
        const uint32_t pb = GP.phase_begin, np = GP.phase_end - pb;
        for (uint32_t i = tid; i < np * (sizeof(TilePhase) / 4); i += kThreads)
            reinterpret_cast<uint32_t*>(sph)[i] = reinterpret_cast<const uint32_t*>(w.phases + pb)[i];
        if (tid < np) {
            const TilePhase& ph = w.phases[pb + tid];
            sboff[tid] = ph.op_end > ph.op_begin ? w.ops[ph.op_begin].data : 0u;
        }
    }
    if (tid == 0) {
        for (int b = 0; b < 3; ++b) {
            mbar_init(&full[b], 1);          // the loading thread's expect_tx arrival
            mbar_init(&staged[b], kCompute); // every compute thread, after its writes
        }
        mbar_init(&mmab[0], 1);
        mbar_init(&mmab[1], 1);
        mbar_init(&aready[0], kCompute);    // every compute thread, after its writes
        mbar_init(&aready[1], kCompute);
        fence_mbar_init();
    }
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_holder;
    const TilePass& P = *sp;
    const uint32_t nph = P.phase_end - P.phase_begin;
    const uint32_t first = sph[0].op_end > sph[0].op_begin ? 0u : 1u;
    const uint32_t last = sph[nph - 1].op_end > sph[nph - 1].op_begin ? nph - 1 : nph - 2;
    const uint32_t m = last - first + 1;           // tensor-core ops per tile

    if (tid >= kMmaWarp) {
        // ---- the MMA warp: one thread issues each slot's MMAs once its A and
        // B are written (slots in whatever order they become ready) ----------
        if (tid == kMmaWarp) {
            const uint64_t mine = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
            uint64_t left[2] = {m * ((mine + 1) / 2), m * (mine / 2)};
            uint32_t ph[2] = {0u, 0u};
            uint64_t last = global_ns();
            uint32_t spins = 0;
            while (left[0] + left[1] > 0) {
                bool did = false;
#pragma unroll
                for (uint32_t s = 0; s < 2; ++s) {
                    if (left[s] && mbar_test(&aready[s], ph[s])) {
                        ph[s] ^= 1u;
                        --left[s];
                        did = true;
                        issue_mmas(mbox[4 * s], mbox[4 * s + 1], mbox[4 * s + 2], &mmab[s]);
                    }
                }
                if (did) {
                    last = global_ns();
                } else if (++spins >= 1024u) {
                    spins = 0;
                    if (global_ns() - last > 2000000000ull) {   // the compute warps stopped: give up
                        atomicExch(err, 5);
                        break;
                    }
                }
            }
        }
    } else if (tid >= kLoadWarp) {
        // ---- HBM traffic: one thread of the load warp, TMA tensor copies -----
        // (the warp's other lanes only wait at the end).  Tile k goes into
        // buffer k % 3 once tile k - 3's staged result has been stored from it
        // (its shared-memory reads done).
        if (tid == kLoadWarp) {
            const CUtensorMap* map = &tmap;
            const uint64_t mine = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
            const uint32_t copies = 1u << geom.n_rem;
            bool ok = true;
            auto store = [&](uint64_t k) -> bool {
                const uint32_t b = static_cast<uint32_t>(k % kBufs);
                if (!mbar_wait_bounded(&staged[b], static_cast<uint32_t>(k / kBufs) & 1u)) return false;
                const uint64_t tile = blockIdx.x + k * gridDim.x;
                const uint32_t src = smem_u32(bufs + b * kBufBytes);
                for (uint32_t cpy = 0; cpy < copies; ++cpy) {
                    int c[5];
                    tile_coords(P, geom, tile, cpy, c);
                    tma_store_5d(map, c, src + cpy * geom.box_bytes);
                }
                bulk_commit();
                return true;
            };
            for (uint64_t k = 0; k < mine && ok; ++k) {
                const uint32_t b = static_cast<uint32_t>(k % kBufs);
                if (k >= kBufs) {
                    ok = store(k - kBufs);
                    bulk_wait_read();        // the buffer has been read out
                    if (!ok) break;
                }
                const uint64_t tile = blockIdx.x + k * gridDim.x;
                const uint32_t dst = smem_u32(bufs + b * kBufBytes);
                mbar_arrive_expect_tx(&full[b], kBufBytes);
                for (uint32_t cpy = 0; cpy < copies; ++cpy) {
                    int c[5];
                    tile_coords(P, geom, tile, cpy, c);
                    tma_load_5d(dst + cpy * geom.box_bytes, map, c, &full[b]);
                }
            }
            for (uint64_t k = mine > kBufs ? mine - kBufs : 0; k < mine && ok; ++k) ok = store(k);
            bulk_wait_all();
            if (!ok) atomicExch(err, 4);
        }
    } else {
        // ---- the compute warps: two slots, one step each per round -----------
        const uint32_t t = tid;
        const uint32_t wq = t >> 5;
        const uint32_t drow = ((wq & 3u) * 32u) << 16 | ((wq >> 2) * 128u);   // lane quarter, M-block
        uint32_t kk[2] = {0u, 1u};
        int jj[2] = {0, -static_cast<int>((m + 1u) / 2u)};
        uint32_t uses[2] = {0u, 0u};
        bool pending[2] = {false, false};
        bool failed = false;
        const float2* __restrict__ mats = w.mats;
        for (;;) {
            bool active = false;
#pragma unroll 1
            for (uint32_t s = 0; s < 2 && !failed; ++s) {
                const uint64_t tile = blockIdx.x + static_cast<uint64_t>(kk[s]) * gridDim.x;
                if (tile >= ntiles) continue;
                active = true;
                if (jj[s] < 0) {
                    ++jj[s];
                    continue;
                }
                const uint32_t j = static_cast<uint32_t>(jj[s]);
                const uint32_t b = kk[s] % kBufs;
                unsigned char* buf = bufs + b * kBufBytes;
                unsigned char* bs = bstage + s * kTcBBytes;
                const uint32_t dcol = tmem + 256u * s;
                // B of the op this step issues (L2-resident; its load latency
                // hides behind the wait and the conversion)
                uint4 bq[kBPerThread];
                if (j < m) {
                    const uint4* bsrc = reinterpret_cast<const uint4*>(mats + sboff[first + j]);
#pragma unroll
                    for (uint32_t i = 0; i < kBPerThread; ++i) bq[i] = __ldg(bsrc + i * kCompute + t);
                }
                if (j == 0) {
                    // the loaded tile -> A of the first op
                    const bool ok = mbar_wait_bounded(&full[b], (kk[s] / kBufs) & 1u);
                    if (compute_any(!ok)) {
                        failed = true;
                        if (t == 0) atomicExch(err, 1);
                        break;
                    }
                    const TilePhase& R = sph[0];
                    uint32_t tp = 0, e[kRegQubits];
#pragma unroll
                    for (int i = 0; i < kThreadQubits; ++i)
                        if ((t >> i) & 1u) tp |= 1u << R.thr_pos[i];
#pragma unroll
                    for (int i = 0; i < kRegQubits; ++i) e[i] = 1u << R.reg_pos[i];
                    const float2* src = reinterpret_cast<const float2*>(buf);
                    float2 v[32];
#pragma unroll
                    for (int r = 0; r < 32; ++r) {
                        uint32_t l = tp;
#pragma unroll
                        for (int i = 0; i < kRegQubits; ++i)
                            if ((r >> i) & 1) l |= e[i];
                        v[r] = src[l];
                    }
                    compute_sync();      // every thread has read the tile: the buffer becomes A
                    if (first == 0) {
                        tc_write_a(v, buf, buf + 32768u);   // own row, identity K order
                    } else {
                        const TilePhase& F = sph[first];
                        uint32_t thr = 0, d[kRegQubits];
#pragma unroll
                        for (int i = 0; i < kThreadQubits; ++i)
                            if ((t >> i) & 1u) thr ^= F.a_thr[i];
#pragma unroll
                        for (int i = 0; i < kRegQubits; ++i) d[i] = F.a_reg[i];
                        float2 h0[16], h1[16];
#pragma unroll
                        for (int c = 0; c < 16; ++c) {
                            h0[c] = v[c];
                            h1[c] = v[16 + c];
                        }
                        scatter16(h0, 0u, thr, d, buf);
                        scatter16(h1, 16u, thr, d, buf);
                    }
                } else {
                    const bool ok = mbar_wait_bounded(&mmab[s], uses[s] & 1u);
                    ++uses[s];
                    pending[s] = false;
                    if (compute_any(!ok)) {
                        failed = true;
                        if (t == 0) atomicExch(err, 2);
                        break;
                    }
                    tc_fence_after();
                    if (j == m) {
                        // the last op's result, staged in its (now free) buffer
                        // in tile order for the TMA store
                        const TilePhase& L = sph[last];
                        uint32_t lt = 0, le[kRegQubits];
#pragma unroll
                        for (int i = 0; i < kThreadQubits; ++i)
                            if ((t >> i) & 1u) lt |= 1u << L.thr_pos[i];
#pragma unroll
                        for (int i = 0; i < kRegQubits; ++i) le[i] = 1u << L.reg_pos[i];
                        float2* dst = reinterpret_cast<float2*>(buf);
#pragma unroll
                        for (uint32_t h = 0; h < 2; ++h) {
                            float2 a[16];
                            read_half(dcol + drow, h, a);
#pragma unroll
                            for (uint32_t c = 0; c < 16; ++c) {
                                const uint32_t r = 16u * h + c;
                                uint32_t l = lt;
#pragma unroll
                                for (int i = 0; i < kRegQubits; ++i)
                                    if ((r >> i) & 1u) l |= le[i];
                                dst[l] = a[c];
                            }
                        }
                        fence_proxy_async();     // generic writes -> the TMA store's reads
                        tc_fence_before();
                        mbar_arrive(&staged[b]);
                        kk[s] += 2;
                        jj[s] = 0;
                        continue;
                    }
                    // D of op j - 1 -> A of op j
                    const TilePhase& F = sph[first + j];
                    uint32_t thr = 0, d[kRegQubits];
#pragma unroll
                    for (int i = 0; i < kThreadQubits; ++i)
                        if ((t >> i) & 1u) thr ^= F.a_thr[i];
#pragma unroll
                    for (int i = 0; i < kRegQubits; ++i) d[i] = F.a_reg[i];
#pragma unroll
                    for (uint32_t h = 0; h < 2; ++h) {
                        float2 a[16];
                        read_half(dcol + drow, h, a);
                        scatter16(a, 16u * h, thr, d, buf);
                    }
                }
                // B into this slot's staging (its previous MMAs are done), then
                // A and B go to the tensor core: the MMA warp issues once every
                // compute thread has arrived
                uint4* bdst = reinterpret_cast<uint4*>(bs);
#pragma unroll
                for (uint32_t i = 0; i < kBPerThread; ++i) bdst[i * kCompute + t] = bq[i];
                if (t == 0) {
                    mbox[4 * s] = smem_u32(buf);
                    mbox[4 * s + 1] = smem_u32(bs);
                    mbox[4 * s + 2] = dcol;
                }
                fence_proxy_async();
                tc_fence_before();
                mbar_arrive(&aready[s]);
                pending[s] = true;
                jj[s] = static_cast<int>(j) + 1;
            }
            if (!active || failed) break;
        }
        // MMAs still in flight (only after a failure) complete before the
        // tensor memory is released
        for (uint32_t s = 0; s < 2; ++s)
            if (pending[s]) mbar_wait_bounded(&mmab[s], uses[s] & 1u);
    }
    // The load and MMA warps ran one thread's code: reconverge each warp
    // before the block-wide barrier, whose aligned form needs whole warps.
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

}  // namespace

// The tile's TMA geometry and tensor map over `state` (see ChainGeom).
static bool chain_tensor_map(const TilePass& P, uint32_t n, float2* state, CUtensorMap* map, ChainGeom* g) {
    // runs of consecutive memory qubits, at most 8 long (a box side is <= 256)
    uint32_t run_lo[kTileQubits], run_len[kTileQubits], nr = 0;
    for (int i = 0; i < kTileQubits;) {
        uint32_t len = 1;
        while (i + static_cast<int>(len) < kTileQubits && len < 8 && P.tile_pos[i + len] == P.tile_pos[i] + len) ++len;
        run_lo[nr] = P.tile_pos[i];
        run_len[nr++] = len;
        i += static_cast<int>(len);
    }
    const uint32_t nd = nr < 5 ? nr : 5;     // real dimensions
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
    *g = ChainGeom{};
    uint32_t boxed = 0;
    for (uint32_t d = 0; d < 5; ++d) {
        if (d < nd) {
            g->lo[d] = static_cast<uint8_t>(run_lo[d]);
            const uint32_t hi = (d + 1 < nd) ? run_lo[d + 1] : n;
            dims[d] = cuuint64_t{1} << (hi - run_lo[d]);
            box[d] = 1u << run_len[d];
            boxed += run_len[d];
        } else {
            g->lo[d] = 64;
            dims[d] = 1;
            box[d] = 1;
        }
        if (d > 0) strides[d - 1] = d < nd ? cuuint64_t{8} << run_lo[d] : cuuint64_t{8} << n;
    }
    g->n_rem = 0;
    for (uint32_t r = nd; r < nr; ++r)
        for (uint32_t k = 0; k < run_len[r]; ++k) g->rem_q[g->n_rem++] = static_cast<uint8_t>(run_lo[r] + k);
    g->box_bytes = 8u << boxed;
    if (boxed + g->n_rem != static_cast<uint32_t>(kTileQubits) || run_lo[0] != 0) return false;
    // the driver's encoder, looked up through the runtime (no link-time
    // dependency on the driver library, which hosts without a GPU lack)
    static PFN_cuTensorMapEncodeTiled encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
    }
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, state, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

cudaError_t launch_chain_pass(float2* state, uint32_t n, const TilePass& host_pass, const TilePass* d_passes,
                              const TilePhase* d_phases, const TileOp* d_ops, const float2* d_mats,
                              uint32_t pass_index, int* err, cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(k_tc_chain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(kSmemChain));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    CUtensorMap map;
    ChainGeom geom;
    if (!chain_tensor_map(host_pass, n, state, &map, &geom)) return cudaErrorInvalidValue;
    const uint64_t tiles = uint64_t{1} << (n - kTileQubits);
    uint64_t grid = static_cast<uint64_t>(sm_count());
    if (grid > tiles) grid = tiles;
    const TileWork w{state, 0, d_passes, d_phases, d_ops, d_mats, pass_index, 0};
    k_tc_chain<<<static_cast<unsigned>(grid), kThreads, kSmemChain, s>>>(map, geom, w, tiles, err);
    return cudaGetLastError();
}

}  // namespace qlb

// chain.cu -- the tensor-core chain kernel: one launch per chain pass.
//
// A chain pass is a tile pass whose register phases each hold one op, a
// 32 x 32 complex unitary on the phase's five register qubits applied by
// tcgen05 split-bf16 MMAs (A = the tile, 256 rows; B = the unitary's real
// embedding, hi/lo; FP32 accumulate in tensor memory; the operand layouts
// are the general tile kernel's, tile.cu).  Between two ops the tile never
// visits the register file longer than one conversion: tensor memory ->
// registers (FP32) -> bf16 hi/lo -> the next op's A operand in shared
// memory, scattered by the planner's per-bit XOR offsets.
//
// Where the general kernel runs one tile at a time and waits for every
// MMA, this one keeps two tiles in flight per SM ("slots", each with 256
// tensor-memory columns and its own B staging): while slot 0's MMAs run,
// the 256 compute threads convert slot 1's tile, and the other way round.
// Slot 1 starts half a tile behind slot 0, so its buffer's next load has
// time to land.  Four producer warps move the tiles between HBM and three
// 64 KB buffers: 16-byte cp.async pieces (TMA bulk copies for runs of
// >= 4 KB) into a buffer, and, after the last op, the result that the
// compute warps staged in the buffer (bank-swizzled tile order) back to
// HBM with 16-byte stores; then the buffer takes the tile three ahead.  A
// thirteenth warp issues the MMAs: a slot's 256 threads arrive on its "A ready"
// barrier after writing A and B and go on to the other slot at once, so an
// MMA issue that waits for the tensor pipe to drain the other slot's MMAs
// stalls nobody.  HBM traffic: 16 B per amplitude per pass.  The store of
// a circuit's last pass also applies its deferred CZ-like sign terms (the
// pass's post terms: a sign per amplitude from its memory index).
//
// The compute warps meet at one CTA barrier per tile (before the loaded
// tile becomes A); otherwise only the MMA dependency orders them, so a warp
// that is ahead converts the other slot while the last one finishes.
//
// Every wait is bounded (2 s / 2^26 polls); on expiry the CTA raises *err,
// waits (bounded) for its own MMAs and copies, frees its tensor memory and
// returns.  A compute thread's wait that gives up is voted on at the next
// per-tile barrier, so all compute threads leave together.
#include "common.cuh"
#include "tc_ptx.cuh"
#include "tile.h"

namespace qlb {

namespace {

using namespace ptx;

constexpr int kCompute = 256;                     // thread t converts A / D row t
constexpr int kProducerWarps = 4;                // warps 8..11: HBM <-> buffers
constexpr int kProducers = 32 * kProducerWarps;
constexpr int kMmaThread = kCompute + kProducers; // warp 12, first lane: MMA issue
// 416 threads, 128 registers a thread (no spills; 13 warps put four on one
// SM sub-partition, whose 16,384 registers cap a thread at 128 -- a build
// at 137 was refused at launch).  Measured on the fused
// 30-qubit circuit: four producer warps 0.7 % faster than three (at 143
// registers), five 0.4 % slower than three; seven, or two compute threads
// per row (at 80 registers), ran no faster.
constexpr int kThreads = kCompute + kProducers + 32;
constexpr uint32_t kTile = 1u << kTileQubits;
constexpr uint32_t kBufBytes = kTile * 8u;        // 64 KB: the tile (fp32) or its A operand (bf16 hi | lo)
constexpr uint32_t kBufs = 3;
constexpr uint32_t kBulkMin = 9;                  // runs of >= 2^9 amplitudes load by bulk copies
constexpr size_t kOffB = size_t{kBufs} * kBufBytes;
constexpr size_t kOffRow = kOffB + 2 * kTcBBytes;                   // u64[128]: memory offset of piece row c
constexpr size_t kOffPass = kOffRow + 128 * 8;
constexpr size_t kOffPhases = kOffPass + sizeof(TilePass);
constexpr size_t kOffBoff = kOffPhases + kMaxSmemPhases * sizeof(TilePhase);
constexpr size_t kOffBar = (kOffBoff + kMaxSmemPhases * 4 + 7) & ~size_t{7};
// mbarriers: full[3], staged[3], mma[2], aready[2]; then the tensor-memory
// address and the two slots' MMA mailboxes (A, B, D addresses)
constexpr size_t kSmemChain = kOffBar + 10 * 8 + 8 + 2 * 16;
static_assert(sizeof(TilePass) % 8 == 0 && sizeof(TilePhase) % 4 == 0, "descriptor staging");
static_assert(kSmemChain <= 227 * 1024, "shared memory per CTA");
constexpr uint32_t kBPerThread = kTcBBytes / (16u * kCompute);   // 4 x 16 B of B per thread
constexpr uint32_t kTmemCols = 512;               // two slots x 2 M-blocks x 128 columns (D: the first 64)

__device__ __forceinline__ uint64_t tile_base(const TilePass& P, uint64_t tile) {
    uint64_t base = 0;
    for (uint32_t j = 0; j < P.n_out; ++j, tile >>= 1)
        if (tile & 1u) base |= uint64_t{1} << P.out_mem[j];
    return base;
}

__device__ __forceinline__ uint32_t fold4(uint32_t i) { return ((i >> 4) ^ (i >> 8) ^ (i >> 12)) & 15u; }

// Barrier 2 over the 96 producer threads.
__device__ __forceinline__ void producer_sync() { asm volatile("bar.sync 2, %0;" ::"n"(kProducers) : "memory"); }
__device__ __forceinline__ bool producer_any(bool x) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 2, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(x ? 1u : 0u), "n"(kProducers)
        : "memory");
    return r != 0;
}

// Barrier 1 over the 256 compute threads (the producer and MMA warps never
// join it), with an OR vote.
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

// Issues the 24 MMAs of one op on A at `a` (hi; lo 32 KB above), B at `b`
// (B_hi; B_lo 8 KB above: N rows 64..127 of the staged image), D at
// tensor-memory column `d`: per M-block of 128 rows and K step, A_hi x B_hi,
// A_hi x B_lo and A_lo x B_hi (N = 64), all accumulated into one D, so the
// read-back is one FP32 value per word.  (Issuing A_hi x [B_hi | B_lo] as
// one N = 128 MMA takes 16 MMAs but leaves two partial sums, D1 | D2, for
// the compute threads to load and add: twice the tensor-memory loads.)
__device__ __forceinline__ void issue_mmas(uint32_t a, uint32_t b, uint32_t d, uint64_t* bar) {
    tc_fence_after();   // after the wait that saw A and B written (and the previous D read)
#pragma unroll
    for (uint32_t mb = 0; mb < 2; ++mb) {
        const uint32_t dm = d + mb * 128u;
#pragma unroll
        for (uint32_t s = 0; s < 4; ++s) {
            const uint64_t ahi = umma_desc_a(a + mb * 16384u + s * 32u);
            tc_mma(dm, ahi, umma_desc_b(b + s * 256u), kTcIdesc64, s > 0 ? 1u : 0u);
            tc_mma(dm, ahi, umma_desc_b(b + 8192u + s * 256u), kTcIdesc64, 1u);
            tc_mma(dm, umma_desc_a(a + 32768u + mb * 16384u + s * 32u), umma_desc_b(b + s * 256u), kTcIdesc64, 1u);
        }
    }
    tc_commit(bar);
}

// tcgen05.wait::ld with the awaited registers as operands, so that no use
// of them is scheduled above the wait.
__device__ __forceinline__ void tmem_wait(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

// This thread's D row (32 amplitudes, columns 0..63 from `col`) in four
// quarters of 8 amplitudes (register indices 8 h .. 8 h + 7), handed to
// use(a, h).  The next quarter's tensor-memory load is in flight while the
// current one is used.
template <typename F>
__device__ __forceinline__ void read_back(uint32_t col, F&& use) {
    uint32_t ra[16], rb[16];
    auto hand = [&](const uint32_t (&r)[16], uint32_t h) {
        float2 a[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = make_float2(__uint_as_float(r[2 * c]), __uint_as_float(r[2 * c + 1]));
        use(a, h);
    };
    tc_ld_16(col, ra);
    tmem_wait(ra);
    tc_ld_16(col + 16u, rb);
    hand(ra, 0u);
    tmem_wait(rb);
    tc_ld_16(col + 32u, ra);
    hand(rb, 1u);
    tmem_wait(ra);
    tc_ld_16(col + 48u, rb);
    hand(ra, 2u);
    tmem_wait(rb);
    hand(rb, 3u);
}

// Scatters amplitudes with register indices base_r .. base_r + N - 1 into
// the A operand at `a` (hi; lo 32 KB above): byte offset = thread part ^
// XOR of d[i] over the index's set bits.
template <int N>
__device__ __forceinline__ void scatter(const float2 (&v)[N], uint32_t base_r, uint32_t thr_off,
                                        const uint32_t (&d)[kRegQubits], unsigned char* a) {
    // Gray-code order: one XOR moves the offset to the next amplitude, so no
    // table of N offsets stays live
    uint32_t off = thr_off;
#pragma unroll
    for (int i = 0; i < kRegQubits; ++i)
        if ((base_r >> i) & 1u) off ^= d[i];
#pragma unroll
    for (uint32_t k = 0; k < N; ++k) {
        if (k) off ^= d[(k & 1u) ? 0 : (k & 2u) ? 1 : (k & 4u) ? 2 : (k & 8u) ? 3 : 4];   // lowest set bit of k
        const uint32_t c = k ^ (k >> 1);
        uint32_t hi, lo;
        tc_split(v[c], hi, lo);
        *reinterpret_cast<uint32_t*>(a + off) = hi;
        *reinterpret_cast<uint32_t*>(a + 32768u + off) = lo;
    }
}

__global__ void __launch_bounds__(kThreads, 1)
k_tc_chain(TileWork w, uint64_t ntiles, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* bufs = smem;
    unsigned char* bstage = smem + kOffB;
    uint64_t* rowoff = reinterpret_cast<uint64_t*>(smem + kOffRow);
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
        // piece rows: 16-byte piece i = l + 32 c of a tile holds tile-local
        // amplitudes 2 i, 2 i + 1 (bits 1..5 from l, 6..12 from c); rowoff[c]
        // is the memory offset of c's bits
        if (tid < 128) {
            uint64_t o = 0;
            for (int i = 0; i < 7; ++i)
                if ((tid >> i) & 1u) o |= uint64_t{1} << GP.tile_pos[6 + i];
            rowoff[tid] = o;
        }
    }
    if (tid == 0) {
        for (int b = 0; b < 3; ++b) {
            mbar_init(&full[b], kProducers);    // one (deferred) arrival per producer thread
            mbar_init(&staged[b], kCompute / 32);   // every compute warp, after its writes
        }
        mbar_init(&mmab[0], 1);
        mbar_init(&mmab[1], 1);
        mbar_init(&aready[0], kCompute / 32);
        mbar_init(&aready[1], kCompute / 32);
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
    const uint64_t mine = blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (tid >= kMmaThread) {
        // ---- the MMA warp: its first thread issues each slot's MMAs once the
        // slot's A and B are written, slots in whichever order they get ready
        if (tid == kMmaThread) {
            uint64_t left[2] = {m * ((mine + 1) / 2), m * (mine / 2)};
            uint32_t ph[2] = {0u, 0u};
            uint64_t last_ns = global_ns();
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
                    last_ns = global_ns();
                } else if (++spins >= 1024u) {
                    spins = 0;
                    if (global_ns() - last_ns > 2000000000ull) {   // the compute warps stopped: give up
                        atomicExch(err, 5);
                        break;
                    }
                }
            }
        }
    } else if (tid >= kCompute) {
        // ---- the producer warps: tile k goes into buffer k % 3 after tile
        // k - 3's staged result has been stored from it ------------------------
        const uint32_t pt = tid - kCompute;            // 0 .. kProducers - 1
        const uint32_t lane = pt & 31u, pw = pt >> 5;  // warp pw takes piece rows c = pw, pw + 7, ...
        const uint32_t nl = P.n_low;
        float2* __restrict__ state = w.state;
        uint64_t gl = 0;
#pragma unroll
        for (int i = 0; i < 5; ++i)
            if ((lane >> i) & 1u) gl |= uint64_t{1} << P.tile_pos[1 + i];
        uint64_t tilemem = 0;                          // memory bits of the tile qubits
        for (int j = 0; j < kTileQubits; ++j) tilemem |= uint64_t{1} << P.tile_pos[j];
        bool ok = true;
        auto store = [&](uint64_t k) -> bool {
            const uint32_t b = static_cast<uint32_t>(k % kBufs);
            const bool got = mbar_wait_bounded(&staged[b], static_cast<uint32_t>(k / kBufs) & 1u);
            if (producer_any(!got)) return false;
            // piece i = lane + 32 c (amplitudes 2 i, 2 i + 1) sits in 16-byte
            // unit i ^ (F >> 1) of the staged layout, halves swapped when F is
            // odd, F = fold4(2 i) = fold4(2 lane) ^ fold4(64 c)
            const uint64_t g0 = tile_base(P, blockIdx.x + k * gridDim.x) | gl;
            const uint4* src = reinterpret_cast<const uint4*>(bufs + b * kBufBytes);
            uint4* dst = reinterpret_cast<uint4*>(state);
            const uint32_t fl = fold4(2u * lane);
            const uint32_t np = P.post_n;
            if (np == 0) {
#pragma unroll 6
                for (uint32_t c = pw; c < 128; c += kProducerWarps) {
                    const uint32_t f = fl ^ fold4(64u * c);
                    uint4 v = src[(lane + 32u * c) ^ (f >> 1)];
                    if (f & 1u) v = make_uint4(v.z, v.w, v.x, v.y);
                    dst[(g0 | rowoff[c]) >> 1] = v;     // amplitudes g, g + 1 (g even)
                }
            } else {
                // the circuit's last pass: its sign terms (CZ-like) flip sign
                // bits on the way out.  Piece i = lane + 32 c holds tile-local
                // amplitudes L = 2 lane + 64 c (+ 1): a term whose out-of-tile
                // and lane bits this thread's tile has fires for the pieces
                // whose row and bit 0 hold the rest of its tile-local mask.
                uint32_t need[kPostMax], s0m[kPostMax];
#pragma unroll
                for (uint32_t i = 0; i < kPostMax; ++i) {
                    need[i] = 0xFFFFFFFFu;      // never met: L < 2^13
                    s0m[i] = 0u;
                    if (i < np) {
                        const uint32_t* r = reinterpret_cast<const uint32_t*>(w.mats + P.post_data + 4u * i);
                        const uint64_t mask = r[0] | (uint64_t{r[1]} << 32);
                        const uint32_t tl = r[6];
                        if (((mask & ~tilemem) & ~g0) == 0 && ((tl & 0x3Eu) & ~(2u * lane)) == 0) {
                            need[i] = tl & 0x1FC1u;
                            s0m[i] = (tl & 1u) ? 0u : 0x80000000u;
                        }
                    }
                }
#pragma unroll 6
                for (uint32_t c = pw; c < 128; c += kProducerWarps) {
                    const uint32_t f = fl ^ fold4(64u * c);
                    uint4 v = src[(lane + 32u * c) ^ (f >> 1)];
                    if (f & 1u) v = make_uint4(v.z, v.w, v.x, v.y);
                    const uint32_t l1 = 64u * c + 1u;
                    uint32_t s0 = 0u, s1 = 0u;
#pragma unroll
                    for (uint32_t i = 0; i < kPostMax; ++i) {
                        const uint32_t hit = (l1 & need[i]) == need[i] ? 0x80000000u : 0u;
                        s1 ^= hit;
                        s0 ^= hit & s0m[i];
                    }
                    dst[(g0 | rowoff[c]) >> 1] = make_uint4(v.x ^ s0, v.y ^ s0, v.z ^ s1, v.w ^ s1);
                }
            }
            return true;
        };
        for (uint64_t k = 0; k < mine && ok; ++k) {
            const uint32_t b = static_cast<uint32_t>(k % kBufs);
            unsigned char* buf = bufs + b * kBufBytes;
            if (k >= kBufs) {
                ok = store(k - kBufs);
                producer_sync();          // every producer has read the buffer out
                if (!ok) break;
            }
            fence_proxy_async();          // generic reads of the buffer precede the copies into it
            const uint64_t base = tile_base(P, blockIdx.x + k * gridDim.x);
            if (nl >= kBulkMin) {
                const uint32_t chunks = 1u << (kTileQubits - nl);
                const uint32_t bytes = (1u << nl) * 8u;
                if (pt == 0) mbar_arrive_expect_tx(&full[b], kBufBytes);
                for (uint32_t c = pt; c < chunks; c += kProducers) {
                    uint64_t g = base;
                    for (uint32_t j = nl; j < static_cast<uint32_t>(kTileQubits); ++j)
                        if ((c >> (j - nl)) & 1u) g |= uint64_t{1} << P.tile_pos[j];
                    bulk_g2s(buf + (static_cast<size_t>(c) << nl) * 8u, state + g, bytes, &full[b]);
                }
                if (pt != 0) mbar_arrive(&full[b]);
            } else {
                const uint32_t d0 = smem_u32(buf) + 16u * lane;
                const uint64_t g0 = base | gl;
#pragma unroll 6
                for (uint32_t c = pw; c < 128; c += kProducerWarps)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d0 + 512u * c),
                                 "l"(state + (g0 | rowoff[c]))
                                 : "memory");
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[b]))
                             : "memory");
            }
        }
        for (uint64_t k = mine > kBufs ? mine - kBufs : 0; k < mine && ok; ++k) ok = store(k);
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (!ok && pt == 0) atomicExch(err, 4);
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
        int bad = 0;             // the first wait of this thread that gave up (1: tile load, 2: MMA)
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
                // B of the op this step issues (L2-resident), copied straight
                // into the slot's staging once its previous MMAs are done; the
                // copy lands while the tile is converted
                auto copy_b = [&]() {
                    const float2* bsrc = mats + sboff[first + j];
                    const uint32_t bdst = smem_u32(bs) + 16u * t;
#pragma unroll
                    for (uint32_t i = 0; i < kBPerThread; ++i)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(bdst + i * 16u * kCompute),
                                     "l"(bsrc + 2u * (i * kCompute + t))
                                     : "memory");
                };
                if (j == 0) {
                    // the loaded tile -> A of the first op
                    if (!mbar_wait_bounded(&full[b], (kk[s] / kBufs) & 1u) && !bad) bad = 1;
                    copy_b();
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
                    // every thread has read the tile: the buffer becomes A.  The
                    // same barrier is the vote on the waits that gave up since
                    // the last one (a failed wait only leaves garbage in
                    // bounds, so the steps in between ran on): all compute
                    // threads leave together.
                    if (compute_any(bad != 0)) {
                        asm volatile("cp.async.wait_all;" ::: "memory");   // this step's B copy
                        failed = true;
                        if (bad) atomicExch(err, bad);
                        break;
                    }
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
                        scatter<32>(v, 0u, thr, d, buf);
                    }
                } else {
                    // no barrier here: a failed wait is voted on at the next
                    // tile's first step
                    if (!mbar_wait_bounded(&mmab[s], uses[s] & 1u) && !bad) bad = 2;
                    ++uses[s];
                    pending[s] = false;
                    tc_fence_after();
                    if (j == m) {
                        // the last op's result, staged in its (now free) buffer:
                        // amplitude l at 8-byte word l ^ fold4(l) (the fold spreads
                        // a warp's stores over the banks; it leaves bit 0 alone, so
                        // amplitudes 2i, 2i + 1 share a 16-byte unit)
                        const TilePhase& L = sph[last];
                        uint32_t lt = 0, le[kRegQubits];
#pragma unroll
                        for (int i = 0; i < kThreadQubits; ++i)
                            if ((t >> i) & 1u) lt |= 1u << L.thr_pos[i];
                        lt ^= fold4(lt);
#pragma unroll
                        for (int i = 0; i < kRegQubits; ++i) {
                            le[i] = 1u << L.reg_pos[i];
                            le[i] ^= fold4(le[i]);
                        }
                        float2* dst = reinterpret_cast<float2*>(buf);
                        read_back(dcol + drow, [&](const float2 (&a)[8], uint32_t h) {
#pragma unroll
                            for (uint32_t c = 0; c < 8; ++c) {
                                const uint32_t r = 8u * h + c;
                                uint32_t l = lt;
#pragma unroll
                                for (int i = 0; i < kRegQubits; ++i)
                                    if ((r >> i) & 1u) l ^= le[i];
                                dst[l] = a[c];
                            }
                        });
                        tc_fence_before();
                        __syncwarp();
                        if ((t & 31u) == 0) mbar_arrive(&staged[b]);   // for the whole warp
                        kk[s] += 2;
                        jj[s] = 0;
                        continue;
                    }
                    // D of op j - 1 -> A of op j
                    copy_b();
                    const TilePhase& F = sph[first + j];
                    uint32_t thr = 0, d[kRegQubits];
#pragma unroll
                    for (int i = 0; i < kThreadQubits; ++i)
                        if ((t >> i) & 1u) thr ^= F.a_thr[i];
#pragma unroll
                    for (int i = 0; i < kRegQubits; ++i) d[i] = F.a_reg[i];
                    read_back(dcol + drow,
                              [&](const float2 (&a)[8], uint32_t h) { scatter<8>(a, 8u * h, thr, d, buf); });
                }
                // A and B go to the tensor core: the MMA warp issues once every
                // compute thread has arrived
                asm volatile("cp.async.wait_all;" ::: "memory");   // this thread's part of B landed
                if (t == 0) {
                    mbox[4 * s] = smem_u32(buf);
                    mbox[4 * s + 1] = smem_u32(bs);
                    mbox[4 * s + 2] = dcol;
                }
                fence_proxy_async();
                tc_fence_before();
                __syncwarp();
                if ((t & 31u) == 0) mbar_arrive(&aready[s]);   // for the whole warp
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

cudaError_t launch_chain_pass(float2* state, uint32_t n, const TilePass* d_passes, const TilePhase* d_phases,
                              const TileOp* d_ops, const float2* d_mats, uint32_t pass_index, int* err,
                              cudaStream_t s) {
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(k_tc_chain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(kSmemChain));
        if (e != cudaSuccess) return e;
        configured = true;
    }
    const uint64_t tiles = uint64_t{1} << (n - kTileQubits);
    uint64_t grid = static_cast<uint64_t>(sm_count());
    if (grid > tiles) grid = tiles;
    const TileWork w{state, 0, d_passes, d_phases, d_ops, d_mats, pass_index, 0};
    k_tc_chain<<<static_cast<unsigned>(grid), kThreads, kSmemChain, s>>>(w, tiles, err);
    return cudaGetLastError();
}

}  // namespace qlb

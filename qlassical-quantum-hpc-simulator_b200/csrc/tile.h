// tile.h -- the tiled execution path: descriptors shared by the host planner
// (tile.cpp) and the sm_100a tile kernel (tile.cu).
//
// A *pass* is one HBM round trip.  A tile is 2^13 amplitudes whose index
// bits are 13 memory qubits, always including qubits 0..2 (so global
// accesses are runs of >= 64 contiguous bytes, whole DRAM sectors; fewer
// fixed qubits leave more room for the pass's own, hence fewer passes).
// Tile-local positions are the tile's qubits in ascending order; the first
// and last phase put the lanes on positions 0..4 (they need only 0..2).  A
// persistent CTA (256 threads, one per SM) walks the tiles: while it computes
// tile i in registers, tile i+1 streams into a second 64 KB shared-memory
// buffer (TMA bulk copies or cp.async, mbarrier-tracked).  Inside a tile, a thread
// holds 32 amplitudes in registers: five tile qubits are "register qubits"
// (a gate on them is register arithmetic), the other eight index the
// thread.  A *phase* fixes that split; between phases the tile is
// transposed through XOR-swizzled shared memory (bank-conflict free for the
// chosen lane qubits).  The last phase stores to HBM from registers or by
// bulk stores from shared memory.
//
// Diagonal instructions (Z, S, RZ, CZ, CP, diagonal UNITARY) and controls
// never need their qubit in registers: their effect depends only on the
// amplitude's global index, which every thread knows.  So a pass's register
// pressure is only the *targets* of non-diagonal instructions.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

struct qlb_engine;
struct qlb_gate_instr;
struct qlb_pool_view;

namespace qlb {

constexpr int kTileQubits = 13;          // 2^13 amplitudes per tile
constexpr int kRegQubits = 5;            // 32 amplitudes per thread
constexpr int kThreadQubits = 8;         // 256 threads
constexpr int kTileThreads = 1 << kThreadQubits;
constexpr int kLaneLow = 5;              // lanes of the first and last phase: tile positions 0..4
constexpr int kTileLow = 3;              // memory qubits 0..kTileLow-1 are in every tile
constexpr int kTileLowMax = 6;           // a planner may keep up to this many (runs of 2^k amplitudes)
constexpr uint32_t kMaxSmemOps = 160;    // ops of one pass cached in shared memory
constexpr uint32_t kMaxSmemPhases = 24;
constexpr uint32_t kDiagStageWords = 1024; // 16-byte words of DIAG data staged in shared memory (16 KB)

enum TileOpKind : uint8_t {
    TOP_U1 = 1,       // complex 2x2 on register bit r0 (controls: ctrl_reg / ctrl_mem)
    TOP_X = 2,        // controlled bit flip on register bit r0 (X, CX, CCX)
    TOP_SWAP = 3,     // swap register bits r0 < r1 (SWAP, CSWAP with controls)
    TOP_U2 = 4,       // 4x4 on register bits (r0 = matrix bit 0 < r1 = matrix bit 1)
    TOP_DENSE = 5,    // 2^k x 2^k on register bits 0..k-1 (k = 3..5), FP32
    TOP_U1R = 6,      // real 2x2 (m[i].x) on register bit r0 (H, RY)
    TOP_RX = 7,       // [[c, -is], [-is, c]] on r0, c = m[0].x, s = m[0].y
    TOP_CPHASE = 8,   // amplitudes with ctrl_reg/ctrl_mem bits all set *= m[0]
    TOP_DENSE_TC = 9, // k = 5 on register bits 0..4 on the tensor cores
    TOP_DIAG = 11,    // a run of diagonal gates: one phase factor per amplitude (layout below)
    TOP_KRON = 12     // a real 2x2 on each of register bits 0..4 (two records, layout below)
};

// Device dispatch codes: one handler per (kind, register bit / bit pair,
// controlled or not), so the kernel's op loop is a single jump table.
enum TileOpCode : uint16_t {
    OPC_NOP = 0,
    OPC_U1 = 1,          // + r0, uncontrolled
    OPC_U1R = 6,         // + r0
    OPC_RX = 11,         // + r0
    OPC_X = 16,          // + r0
    OPC_U1_CTL = 21,     // + r0, register controls ctrl_reg (any 1-qubit kind, complex m)
    OPC_X_CTL = 26,      // + r0
    OPC_SWAP = 31,       // + pair index of (r0 < r1)
    OPC_U2 = 41,         // + pair index
    OPC_DENSE3 = 51,
    OPC_DENSE4 = 52,
    OPC_DENSE5 = 53,
    OPC_DENSE_TC = 54,
    OPC_DIAG = 55,
    OPC_CPHASE = 56,
    OPC_KRON = 57,
    OPC_COUNT = 58
};
// (a, b), a < b < 5  ->  0..9
__host__ __device__ constexpr uint32_t reg_pair_index(uint32_t a, uint32_t b) { return a * (9u - a) / 2u + (b - a - 1u); }

// One register-level op, 64 bytes (four 16-byte words read with vector loads).
//   TOP_DIAG: data = float2 offset of its tables in the matrix buffer:
//     [flags & 1] R: 32 float2, the factor of each register index (terms on register bits only)
//     [flags & 2] 256 float2, the factor of each thread (terms on the phase's thread bits only)
//     [flags & 4] 256 u32, the sign pattern of each thread (pi terms: register x thread bits)
//     g = (flags >> 8) & 0xFF: g register masks (u32, padded to 16 B), then g tables of
//                 256 float2: thread t multiplies the registers containing mask k by table k[t]
//     n & 0xFFFF  T terms, 32 B each: {u64 mem mask, float2 p1, float2 p0}: a thread whose
//                 index has every mask bit set multiplies by p1, otherwise by p0
//     n >> 16     S terms, 16 B each: {u64 mem mask, u32 register pattern, 0}: sign flips
//     ctrl_reg    G groups: a 16 B header {u32 register mask, u32 count, 0, 0}, then count
//                 terms of 16 B {u64 mem mask, float2 phase}: the amplitudes whose index has
//                 every mem-mask bit and whose register index contains the mask get the phase
//     m[0].x      (u32 bits) 0, or the data's length in 16-byte words when the kernel is to
//                 stage it in shared memory first; the data starts on a 16-byte boundary
//                 and is padded to whole words
//   TOP_KRON: five real 2x2 matrices (m00, m01, m10, m11), one per register bit, in two
//     records: bit 0 in words 2 of this record, bit 1 in its word 3, bits 2, 3, 4 in words
//     1, 2, 3 of the next record (code OPC_NOP, never dispatched: the op's handler skips it)
struct TileOp {
    uint16_t code;          // TileOpCode
    uint8_t kind, k;        // TileOpKind; DENSE: k
    uint8_t r0, r1;
    uint8_t has_mem, pad;   // has_mem: ctrl_mem != 0
    uint32_t ctrl_reg;      // register-bit mask that must be all ones
    uint32_t data;          // U2/DENSE/TC/DIAG: float2 offset into the matrix buffer
    uint32_t flags;
    uint32_t n;
    uint64_t ctrl_mem;      // memory-qubit mask (non-register qubits) that must be all ones
    float2 m[4];            // matrix / coefficients / phase
};
static_assert(sizeof(TileOp) == 64, "TileOp is four 16-byte words");

// TilePhase.flags
constexpr uint8_t kPhaseTcEntry = 1;   // the phase opens with its DENSE_TC op, entered without a transpose

struct TilePhase {
    uint8_t reg_pos[kRegQubits];      // register bit j <- tile-local position
    uint8_t thr_pos[kThreadQubits];   // thread bit j  <- tile-local position (lanes = j < 5)
    uint8_t flags;                    // kPhase* bits
    uint8_t pad[2];
    uint32_t op_begin, op_end;
    // kPhaseTcEntry: the previous phase's registers are written straight into
    // the tensor-core A operand of this phase's layout (the transpose and the
    // operand write in one step).  The byte offset of an amplitude in A is the
    // XOR of a_thr[j] over the set bits j of the previous phase's thread index
    // and of a_reg[j] over the set bits of its previous register index.
    uint16_t a_thr[kThreadQubits];
    uint16_t a_reg[kRegQubits];
    uint16_t pad2[3];
};
static_assert(sizeof(TilePhase) == 56, "TilePhase layout");

struct TilePass {
    uint8_t tile_pos[kTileQubits];    // tile-local position j -> memory qubit (ascending)
    uint8_t n_out;                    // number of non-tile qubits
    uint8_t n_low;                    // tile_pos[j] == j for j < n_low (>= kTileLow): runs of 2^n_low amps
    uint8_t features;                 // kernel features the pass needs (kPass* bits)
    uint8_t out_mem[40];              // non-tile memory qubits, ascending
    uint32_t phase_begin, phase_end;
    // Chain passes only: post_n (<= kPostMax) sign terms applied to every
    // amplitude as the tile is stored, 32 B each at float2 offset post_data of
    // the matrix buffer: {u64 memory mask, float2 p1 = -1, float2 p0 = 1,
    // u32 the mask's tile-local bits, u32 0} -- an amplitude whose memory
    // index has every mask bit set changes sign.
    uint32_t post_data, post_n;
    uint32_t pad[2];
};
static_assert(sizeof(TilePass) == 80, "TilePass layout (16-byte multiple)");
constexpr uint32_t kPostMax = 4;

// Device program of one execute(): all passes, phases, ops, matrices.
struct TileProgram {
    std::vector<TilePass> passes;
    std::vector<TilePhase> phases;
    std::vector<TileOp> ops;
    std::vector<float2> mats;
};

// One entry of a multi-state launch: tiles [tile_begin, tile_begin +
// 2^(n - 13)) of the launch's flattened tile range apply pass `pass` to the
// state at `state` (entries sorted by tile_begin, contiguous).
struct TileWork {
    float2* state;
    uint64_t tile_begin;
    const TilePass* passes;     // the entry's program (its own arrays: states of
    const TilePhase* phases;    // different programs share one launch)
    const TileOp* ops;
    const float2* mats;
    uint32_t pass;              // index into `passes`
    uint32_t pad;
};

// Kernel features of a pass, which pick the kernel body it runs (the
// smallest that holds its ops): tensor-core ops (the CTA allocates tensor
// memory), FP32 DENSE3-5 ops (the largest body), register SWAPs, U2
// register-pair ops, and X, controlled 1-qubit and CPHASE ops (not in the
// tensor-core body).
constexpr int kPassTensorCores = 1;
constexpr int kPassWide = 2;
constexpr int kPassSwaps = 4;
constexpr int kPassPairs = 8;
constexpr int kPassCtl = 16;
// The pass is in chain form (every register phase one tensor-core op): a
// single-state launch runs it on the tensor-core chain kernel (chain.cu).
// Not a body feature: tile_body() ignores it.
constexpr int kPassChain = 32;

// Kernel bodies (instantiations of the tile kernel), smallest first: 1-qubit,
// controlled and diagonal ops; those plus register SWAPs; uncontrolled
// 1-qubit rotations, diagonal, SWAP, U2 and tensor-core ops; everything,
// with the FP32 DENSE3-5 handlers.  A pass runs tile_body(features).
constexpr int kBodyNarrow = 0, kBodySwaps = 1, kBodyTc = 2, kBodyWide = 3;
constexpr int tile_body(int features) {
    return (features & kPassWide) ? kBodyWide
           : (features & (kPassTensorCores | kPassPairs)) ? ((features & kPassCtl) ? kBodyWide : kBodyTc)
           : (features & kPassSwaps) ? kBodySwaps
                                     : kBodyNarrow;
}
// Whether kernel body `body` has a handler for dispatch code `code` (the
// planner checks every op of a pass against the body the pass will run).
constexpr bool tile_body_handles(int body, uint32_t code) {
    const bool common =
        (code >= OPC_U1 && code < OPC_SWAP) || code == OPC_DIAG || code == OPC_CPHASE || code == OPC_KRON;
    const bool swap = code >= OPC_SWAP && code < OPC_U2;
    const bool u2 = code >= OPC_U2 && code < OPC_DENSE3;
    switch (body) {
    case kBodyWide: return code >= OPC_U1 && code < OPC_COUNT;
    case kBodyTc:
        return (code >= OPC_U1 && code < OPC_X) || code == OPC_DIAG || code == OPC_KRON || swap || u2 ||
               code == OPC_DENSE_TC;
    case kBodySwaps: return common || swap;
    default: return common;
    }
}

// `err` (device int) receives a nonzero code if a bounded wait gave up.
// `features`: the pass's kPass* bits (union over the entries of a work list).
cudaError_t launch_tile_pass(float2* state, uint32_t n, const TilePass* d_passes, const TilePhase* d_phases,
                             const TileOp* d_ops, const float2* d_mats, uint32_t pass_index, int features,
                             int* err, cudaStream_t s);
int sm_count();   // multiprocessors of the current device (cached)

// The chain kernel (chain.cu): one launch applies chain pass `pass_index`
// to the state; returns the launch status.
cudaError_t launch_chain_pass(float2* state, uint32_t n, const TilePass* d_passes, const TilePhase* d_phases,
                              const TileOp* d_ops, const float2* d_mats, uint32_t pass_index, int* err,
                              cudaStream_t s);

// Runs the tile kernel's bounded mbarrier wait on a barrier that never
// completes; *err becomes 1 when the wait gives up (as it must).
cudaError_t launch_wait_selftest(uint64_t limit_ns, int* err, cudaStream_t s);

// Sets the tile kernel's shared-memory limit (once per process; call before
// capturing a launch into a CUDA graph).
cudaError_t configure_tile_kernel();
// One launch over a work list in device memory (batched and served states);
// `max_ctas` caps the grid (0: one CTA per SM).  `d_tile_entry` (optional):
// the work-list index of every tile of the launch, which replaces the
// kernel's binary search over the entries' tile_begin.
cudaError_t launch_tile_work(const TileWork* d_work, uint32_t n_work, uint64_t total_tiles, int features, int* err,
                             cudaStream_t s, uint32_t max_ctas = 0, const uint32_t* d_tile_entry = nullptr);

// Host-side helpers shared between engine.cpp and tile.cpp.
struct Layout {
    uint32_t mem[64];
    void reset() {
        for (uint32_t i = 0; i < 64; ++i) mem[i] = i;
    }
};
struct Mat2f;
Mat2f gate_matrix_1q(uint8_t type, float param);
uint32_t instr_qubit(const qlb_gate_instr& in, uint32_t j);
void measure(qlb_engine& e, uint32_t mem_qubit);
// One instruction whose qubits are memory qubits; `mat` is its complex64
// matrix in device memory (UNITARY / FUSED_BLOCK only).
void apply_plain(qlb_engine& e, const qlb_gate_instr& in, const float2* mat);

}  // namespace qlb

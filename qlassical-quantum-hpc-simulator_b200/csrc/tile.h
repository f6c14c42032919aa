// tile.h -- the tiled execution path: descriptors shared by the host planner
// (tile.cpp) and the sm_100a tile kernel (tile.cu).
//
// A *pass* is one HBM round trip: every CTA owns one tile of 2^13
// amplitudes whose index bits are 13 memory qubits (always including qubits
// 0..4, so each warp access is 32 consecutive complex64 = 256 B), runs a
// list of instructions on it, and writes it back.  Inside a pass the tile
// lives in registers: 256 threads x 32 amplitudes.  Five tile qubits are
// "register qubits" (a gate on them is pure register arithmetic), the other
// eight index the thread.  A *phase* fixes that split; between phases the
// tile is transposed through shared memory (64 KB, XOR-swizzled so both the
// write and the read are bank-conflict free).
//
// Diagonal instructions (Z, S, RZ, CZ, CP) and controls never need their
// qubit in registers: their effect depends only on the amplitude's global
// index, which every thread knows.  So a pass's register pressure is only
// the *targets* of non-diagonal instructions.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

struct qlb_engine;
struct qlb_gate_instr;
struct qlb_pool_view;

namespace qlb {

constexpr int kTileQubits = 13;          // 2^13 amplitudes per CTA tile
constexpr int kRegQubits = 5;            // 32 amplitudes per thread
constexpr int kThreadQubits = 8;         // 256 threads
constexpr int kTileThreads = 1 << kThreadQubits;
constexpr int kLaneLow = 5;              // tile positions 0..4 = memory qubits 0..4

enum TileOpKind : uint8_t {
    TOP_U1 = 1,       // 2x2 on register bit r0 (controls: ctrl_reg / ctrl_mem)
    TOP_X = 2,        // controlled bit flip on register bit r0 (X, CX, CCX)
    TOP_SWAP = 3,     // swap register bits r0, r1 (SWAP, CSWAP with controls)
    TOP_U2 = 4,       // 4x4 on register bits (r0 = matrix bit 0, r1 = matrix bit 1)
    TOP_DENSE = 5,    // 2^k x 2^k on register bits 0..k-1 (k = 3..5), FP32
    TOP_PHASE = 6,    // diagonal phase polynomial, terms[data .. data+count)
    TOP_DENSE_TC = 7  // k = 5 on register bits 0..4 on the tensor cores
};

struct TileOp {
    uint8_t kind;
    uint8_t r0, r1, k;
    uint32_t ctrl_reg;      // register-bit mask that must be all ones
    uint64_t ctrl_mem;      // memory-qubit mask (non-register qubits) that must be all ones
    float2 m[4];            // TOP_U1 matrix (row-major)
    uint32_t data;          // TOP_U2/DENSE: float2 offset of the matrix; TOP_PHASE: word offset
    uint32_t count;         // unused (alignment)
};

// A TOP_PHASE op multiplies every amplitude by exp(i*phi(index)) with
//   phi = c + sum_a th_a b_a + sum_{a<b} th_ab b_a b_b    (b_q = index bit q)
// evaluated in fixed point (turns * 2^32, wrapping = mod 2*pi).  For one
// phase the host splits the terms by where their qubits live: both outside
// the registers (thread constant), one in registers (linear in a register
// bit), both in registers (quadratic, uniform).  Layout of the uint32 words
// at op.data:
//   [0] constant, [1..5] unconditional linear coefficient of register bit j,
//   [6..15] quadratic coefficient of register bits (j<k, lexicographic),
//   [16] T = number of thread-constant terms, [17] L = number of linear
//   terms conditioned on a non-register bit, then T pairs
//   (ga | gb << 8, angle) and L pairs (j | gb << 8, angle); gb = 0xFF means
//   "no second qubit".
constexpr uint32_t kPhaseHeaderWords = 18;

struct TilePhase {
    uint8_t reg_pos[kRegQubits];      // register bit j <- tile-local position
    uint8_t thr_pos[kThreadQubits];   // thread bit j  <- tile-local position (lanes = j < 5)
    uint8_t pad[3];
    uint32_t op_begin, op_end;
};

struct TilePass {
    uint8_t tile_pos[kTileQubits];    // tile-local position j -> memory qubit (ascending)
    uint8_t n_out;                    // number of non-tile qubits
    uint8_t out_pos[2];               // unused padding for alignment
    uint8_t out_mem[40];              // non-tile memory qubits, ascending
    uint32_t phase_begin, phase_end;
};

// Device program of one execute(): all passes, phases, ops, terms, matrices.
struct TileProgram {
    std::vector<TilePass> passes;
    std::vector<TilePhase> phases;
    std::vector<TileOp> ops;
    std::vector<uint32_t> pdata;
    std::vector<float2> mats;
};

cudaError_t launch_tile_pass(float2* state, uint32_t n, const TilePass* d_pass, const TilePhase* d_phases,
                             const TileOp* d_ops, const uint32_t* d_pdata, const float2* d_mats,
                             uint32_t pass_index, cudaStream_t s);

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

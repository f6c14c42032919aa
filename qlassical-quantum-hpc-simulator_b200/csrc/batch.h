// batch.h -- many independent states in one device buffer: descriptors
// shared by the batched / served runtimes (batch.cpp, serve.cpp) and their
// kernels (batch.cu, tile.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qlb {

constexpr uint32_t kBatchMinQubits = 13;   // states below one tile are padded to 13 qubits
constexpr uint32_t kBatchMaxQubits = 34;
constexpr uint32_t kBatchStride = 40;      // doubles per state in the <Z> result (last = sum |a|^2)

struct BatchState {
    uint64_t offset;        // float2 offset of the state in the shared buffer
    uint32_t num_qubits;    // the circuit's qubits (<Z> is reported for these)
    uint32_t eff_qubits;    // allocated qubits (>= 13)
};

cudaError_t launch_set_basis(float2* base, const BatchState* st, uint32_t count, cudaStream_t s);
// <Z_q> of every state into out[c * stride + q] (and sum |a|^2 at
// out[c * stride + stride - 1]); chunk_begin[c] = first 2^13-chunk of state
// c (count + 1 entries); `partial` holds batch_partial_doubles(total) doubles.
cudaError_t launch_batch_expect_z(const float2* base, const BatchState* st, uint32_t count,
                                  const uint64_t* chunk_begin, uint64_t total_chunks, double* partial, double* out,
                                  uint32_t stride, cudaStream_t s);
uint64_t batch_partial_doubles(uint64_t total_chunks);

}  // namespace qlb

// batch.cu -- kernels over many independent states at once (batched and
// served circuits): |0...0> set-up and the per-qubit <Z> reduction.
//
// The reduction is deterministic per state: each block reduces one chunk of
// 2^13 amplitudes of one state into 14 partial sums, and one block per state
// adds its chunks' partials in chunk order.  A state's result therefore does
// not depend on which other states share the launch.
#include "batch.h"
#include "common.cuh"

namespace qlb {

namespace {
constexpr unsigned kThreads = 256;
constexpr uint32_t kChunkLog2 = 13;
constexpr uint32_t kPart = 1 + kChunkLog2;   // total + qubits 0..12 of the chunk

__device__ __forceinline__ double p2(float2 a) {
    const double x = a.x, y = a.y;
    return x * x + y * y;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Block-wide sum in a fixed order; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    return t;
}

// Largest i with begin[i] <= x.
__device__ __forceinline__ uint32_t upper_index(const uint64_t* __restrict__ begin, uint32_t count, uint64_t x) {
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (begin[mid] <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_set_basis(float2* __restrict__ base, const BatchState* __restrict__ st, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) base[st[i].offset] = make_float2(1.f, 0.f);
}

// One chunk of one state per block iteration: amplitude t + 256 j of the
// chunk has bits 0..7 = t and bits 8..12 = j.
__global__ void __launch_bounds__(kThreads) k_chunk_marginals(const float2* __restrict__ base,
                                                              const BatchState* __restrict__ st, uint32_t count,
                                                              const uint64_t* __restrict__ chunk_begin,
                                                              uint64_t total_chunks, double* __restrict__ partial) {
    __shared__ double sh[32];
    for (uint64_t g = blockIdx.x; g < total_chunks; g += gridDim.x) {
        const uint32_t c = upper_index(chunk_begin, count, g);
        const uint64_t k = g - chunk_begin[c];
        const float2* a = base + st[c].offset + (k << kChunkLog2);
        double tot = 0.0, jb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
        for (uint32_t j = 0; j < 32; ++j) {
            const double p = p2(a[threadIdx.x + kThreads * j]);
            tot += p;
#pragma unroll
            for (uint32_t b = 0; b < 5; ++b)
                if ((j >> b) & 1u) jb[b] += p;
        }
        double* out = partial + g * kPart;
        double v = block_sum(tot, sh);
        if (threadIdx.x == 0) out[0] = v;
#pragma unroll
        for (uint32_t q = 0; q < 8; ++q) {
            v = block_sum(((threadIdx.x >> q) & 1u) ? tot : 0.0, sh);
            if (threadIdx.x == 0) out[1 + q] = v;
        }
#pragma unroll
        for (uint32_t b = 0; b < 5; ++b) {
            v = block_sum(jb[b], sh);
            if (threadIdx.x == 0) out[1 + 8 + b] = v;
        }
    }
}

// One block per state: <Z_q> = sum|a|^2 - 2 * sum_{bit q set} |a|^2.
__global__ void __launch_bounds__(kThreads) k_finalize_expect_z(const double* __restrict__ partial,
                                                                const BatchState* __restrict__ st,
                                                                const uint64_t* __restrict__ chunk_begin,
                                                                double* __restrict__ out, uint32_t stride) {
    __shared__ double sh[32];
    const uint32_t c = blockIdx.x;
    const uint64_t c0 = chunk_begin[c], nch = chunk_begin[c + 1] - c0;
    const uint32_t nq = st[c].num_qubits;
    double acc[1 + kBatchMaxQubits];
#pragma unroll
    for (uint32_t q = 0; q <= kBatchMaxQubits; ++q) acc[q] = 0.0;
    for (uint64_t k = threadIdx.x; k < nch; k += blockDim.x) {
        const double* p = partial + (c0 + k) * kPart;
        const double tot = p[0];
        acc[0] += tot;
#pragma unroll
        for (uint32_t q = 0; q < kChunkLog2; ++q) acc[1 + q] += p[1 + q];
#pragma unroll
        for (uint32_t q = kChunkLog2; q < kBatchMaxQubits; ++q)
            if ((k >> (q - kChunkLog2)) & 1u) acc[1 + q] += tot;
    }
    const double tot = block_sum(acc[0], sh);
    double* o = out + static_cast<uint64_t>(c) * stride;
#pragma unroll
    for (uint32_t q = 0; q < kBatchMaxQubits; ++q) {
        const double s = block_sum(acc[1 + q], sh);
        if (threadIdx.x == 0 && q < nq) o[q] = tot - 2.0 * s;
    }
    if (threadIdx.x == 0) o[stride - 1] = tot;
}
}  // namespace

cudaError_t launch_set_basis(float2* base, const BatchState* st, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_set_basis<<<(count + kThreads - 1) / kThreads, kThreads, 0, s>>>(base, st, count);
    return cudaGetLastError();
}

cudaError_t launch_batch_expect_z(const float2* base, const BatchState* st, uint32_t count,
                                  const uint64_t* chunk_begin, uint64_t total_chunks, double* partial, double* out,
                                  uint32_t stride, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const uint64_t cap = static_cast<uint64_t>(sm_count()) * 8;
    const unsigned grid = static_cast<unsigned>(total_chunks < cap ? total_chunks : cap);
    k_chunk_marginals<<<grid, kThreads, 0, s>>>(base, st, count, chunk_begin, total_chunks, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_finalize_expect_z<<<count, kThreads, 0, s>>>(partial, st, chunk_begin, out, stride);
    return cudaGetLastError();
}

uint64_t batch_partial_doubles(uint64_t total_chunks) { return total_chunks * kPart; }

}  // namespace qlb

// common.cuh -- device helpers shared by the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace qlb {

// Grid size for grid-stride sweeps: a multiple of the SM count (148 on
// B200) so every SM gets the same number of resident CTAs.
int sm_count();
inline unsigned sweep_grid(uint64_t items, unsigned threads, unsigned ctas_per_sm = 8) {
    uint64_t need = (items + threads - 1) / threads;
    uint64_t cap = static_cast<uint64_t>(sm_count()) * ctas_per_sm;
    if (need < 1) need = 1;
    return static_cast<unsigned>(need < cap ? need : cap);
}

// insert_zero_bit (state_vector_utils.hpp:23-28): a zero at position t.
__host__ __device__ __forceinline__ uint64_t insert_zero_bit(uint64_t idx, uint32_t t) {
    const uint64_t mask = (uint64_t{1} << t) - 1;
    return (idx & mask) | ((idx & ~mask) << 1);
}

// Zeros at the ascending positions h[0..nh-1].
struct Holes {
    uint32_t n;
    uint32_t h[6];
};
__host__ __device__ __forceinline__ uint64_t insert_zero_bits(uint64_t idx, const Holes& hs) {
#pragma unroll
    for (uint32_t j = 0; j < 6; ++j)
        if (j < hs.n) idx = insert_zero_bit(idx, hs.h[j]);
    return idx;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// acc + a*b
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}

}  // namespace qlb

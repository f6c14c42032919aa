// state.cu -- state-vector set-up kernels (CUDAStateVector::initialize).
//
// |0...0> initialisation (cpu_state_vector.hpp:54-78) and the complex128 <->
// complex64 conversions used by initialize(span) (:82-115) and state().
#include "common.cuh"
#include "kernels.h"

namespace qlb {

namespace {
constexpr unsigned kThreads = 256;

__global__ void k_init_zero(float4* __restrict__ a, uint64_t n4) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n4; i += stride)
        a[i] = make_float4(i == 0 ? 1.f : 0.f, 0.f, 0.f, 0.f);
}

__global__ void k_init_zero_small(float2* a, uint64_t dim) {
    for (uint64_t i = 0; i < dim; ++i) a[i] = make_float2(i == 0 ? 1.f : 0.f, 0.f);
}

__global__ void k_c128_to_c64(const double2* __restrict__ src, float2* __restrict__ dst, uint64_t count) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride) {
        double2 v = src[i];
        dst[i] = make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
    }
}

__global__ void k_c64_to_c128(const float2* __restrict__ src, double2* __restrict__ dst, uint64_t count) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride) {
        float2 v = src[i];
        dst[i] = make_double2(v.x, v.y);
    }
}
__global__ void k_gather(const float2* __restrict__ a, const uint64_t* __restrict__ idx, uint64_t count,
                         double2* __restrict__ out) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride) {
        const float2 v = a[idx[i]];
        out[i] = make_double2(v.x, v.y);
    }
}
}  // namespace

cudaError_t launch_gather(const float2* a, const uint64_t* idx, uint64_t count, double2* out, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_gather<<<sweep_grid(count, kThreads), kThreads, 0, s>>>(a, idx, count, out);
    return cudaGetLastError();
}

cudaError_t launch_init_zero(float2* a, uint64_t dim, cudaStream_t s) {
    if (dim == 0) return cudaErrorInvalidValue;
    if (dim <= 2) {
        k_init_zero_small<<<1, 1, 0, s>>>(a, dim);
    } else {
        const uint64_t n4 = dim / 2;
        k_init_zero<<<sweep_grid(n4, kThreads), kThreads, 0, s>>>(reinterpret_cast<float4*>(a), n4);
    }
    return cudaGetLastError();
}

cudaError_t launch_c128_to_c64(const double2* src, float2* dst, uint64_t count, cudaStream_t s) {
    k_c128_to_c64<<<sweep_grid(count, kThreads), kThreads, 0, s>>>(src, dst, count);
    return cudaGetLastError();
}

cudaError_t launch_c64_to_c128(const float2* src, double2* dst, uint64_t count, cudaStream_t s) {
    k_c64_to_c128<<<sweep_grid(count, kThreads), kThreads, 0, s>>>(src, dst, count);
    return cudaGetLastError();
}

}  // namespace qlb

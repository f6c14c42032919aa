// gates.cu -- plain per-instruction kernels: one HBM sweep per instruction.
//
// Each kernel is the sm_100a counterpart of one reference loop
// (cpu_openmp_engine.hpp): single_target_loop (:260-266) for the 2x2 gates,
// double/triple_hole_loop (:270-334) for CX/SWAP/CCX/CSWAP, apply_unitary
// (:539-606) for dense k-qubit matrices.  They are HBM-bound: 16 B per
// touched amplitude (8 B read + 8 B write of complex64).  Amplitude pairs
// that share bit 0 are moved as one 16-byte float4 so every warp request is
// a full 512-byte coalesced transaction.
#include "common.cuh"
#include "kernels.h"

namespace qlb {

namespace {

constexpr unsigned kThreads = 256;

__device__ __forceinline__ void u1_pair(float2& a0, float2& a1, const Mat2f& m) {
    float2 o0 = cmul(m.m[0], a0);
    o0 = cfma(m.m[1], a1, o0);
    float2 o1 = cmul(m.m[2], a0);
    o1 = cfma(m.m[3], a1, o1);
    a0 = o0;
    a1 = o1;
}

// Target t >= 1: item k covers amplitudes i0, i0+1 (bit t = 0) and their
// partners i0|2^t, i0+1|2^t.
__global__ void __launch_bounds__(kThreads) k_u1_hi(float2* __restrict__ a, uint64_t items, uint32_t t, Mat2f m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        const uint64_t i0 = insert_zero_bit(2 * k, t);
        const uint64_t i1 = i0 | (uint64_t{1} << t);
        float4 x = *reinterpret_cast<const float4*>(a + i0);
        float4 y = *reinterpret_cast<const float4*>(a + i1);
        float2 x0 = make_float2(x.x, x.y), x1 = make_float2(x.z, x.w);
        float2 y0 = make_float2(y.x, y.y), y1 = make_float2(y.z, y.w);
        u1_pair(x0, y0, m);
        u1_pair(x1, y1, m);
        *reinterpret_cast<float4*>(a + i0) = make_float4(x0.x, x0.y, x1.x, x1.y);
        *reinterpret_cast<float4*>(a + i1) = make_float4(y0.x, y0.y, y1.x, y1.y);
    }
}

// Target t == 0: the pair is one float4.
__global__ void __launch_bounds__(kThreads) k_u1_lo(float2* __restrict__ a, uint64_t items, Mat2f m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        float4 x = reinterpret_cast<const float4*>(a)[k];
        float2 a0 = make_float2(x.x, x.y), a1 = make_float2(x.z, x.w);
        u1_pair(a0, a1, m);
        reinterpret_cast<float4*>(a)[k] = make_float4(a0.x, a0.y, a1.x, a1.y);
    }
}

// diag(d0, d1) on target t; `only_one` touches only the bit-t = 1 half.
__global__ void __launch_bounds__(kThreads) k_diag1(float2* __restrict__ a, uint64_t items, uint32_t t,
                                                     float2 d0, float2 d1, int only_one) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        if (only_one) {  // t >= 1: item = two consecutive amplitudes of the |1> half
            const uint64_t i1 = insert_zero_bit(2 * k, t) | (uint64_t{1} << t);
            float4 x = *reinterpret_cast<const float4*>(a + i1);
            float2 p = cmul(d1, make_float2(x.x, x.y)), q = cmul(d1, make_float2(x.z, x.w));
            *reinterpret_cast<float4*>(a + i1) = make_float4(p.x, p.y, q.x, q.y);
        } else {  // full sweep, item = float4 at 2k
            float4 x = reinterpret_cast<const float4*>(a)[k];
            const uint64_t i = 2 * k;
            float2 f0 = ((i >> t) & 1) ? d1 : d0;
            float2 f1 = (((i + 1) >> t) & 1) ? d1 : d0;
            float2 p = cmul(f0, make_float2(x.x, x.y)), q = cmul(f1, make_float2(x.z, x.w));
            reinterpret_cast<float4*>(a)[k] = make_float4(p.x, p.y, q.x, q.y);
        }
    }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) k_swap_subspace(float2* __restrict__ a, uint64_t items, Holes hs,
                                                             uint64_t ma, uint64_t mb) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        if (VEC) {
            const uint64_t base = insert_zero_bits(2 * k, hs);
            float4* pa = reinterpret_cast<float4*>(a + (base | ma));
            float4* pb = reinterpret_cast<float4*>(a + (base | mb));
            float4 x = *pa, y = *pb;
            *pa = y;
            *pb = x;
        } else {
            const uint64_t base = insert_zero_bits(k, hs);
            float2 x = a[base | ma], y = a[base | mb];
            a[base | ma] = y;
            a[base | mb] = x;
        }
    }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads) k_phase_mask(float2* __restrict__ a, uint64_t items, Holes hs,
                                                          uint64_t mask, float2 ph) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        if (VEC) {
            float4* p = reinterpret_cast<float4*>(a + (insert_zero_bits(2 * k, hs) | mask));
            float4 x = *p;
            float2 u = cmul(ph, make_float2(x.x, x.y)), v = cmul(ph, make_float2(x.z, x.w));
            *p = make_float4(u.x, u.y, v.x, v.y);
        } else {
            const uint64_t i = insert_zero_bits(k, hs) | mask;
            a[i] = cmul(ph, a[i]);
        }
    }
}

// Dense 2^K x 2^K complex64 matrix, one group of 2^K amplitudes per thread
// iteration; the matrix sits in shared memory and is read as broadcasts.
struct Offsets {
    uint64_t o[64];
};

template <int K>
__global__ void __launch_bounds__(128) k_dense(float2* __restrict__ a, uint64_t groups, Holes hs, Offsets off,
                                               const float2* __restrict__ mat) {
    constexpr int D = 1 << K;
    __shared__ float2 M[D * D];
    for (int i = threadIdx.x; i < D * D; i += blockDim.x) M[i] = mat[i];
    __syncthreads();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g < groups; g += stride) {
        const uint64_t base = insert_zero_bits(g, hs);
        float2 v[D];
#pragma unroll
        for (int j = 0; j < D; ++j) v[j] = a[base | off.o[j]];
#pragma unroll 1
        for (int r = 0; r < D; ++r) {
            float2 acc = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < D; ++c) acc = cfma(M[r * D + c], v[c], acc);
            a[base | off.o[r]] = acc;
        }
    }
}

Holes make_holes(const uint32_t* h, uint32_t nh) {
    Holes hs{};
    hs.n = nh;
    for (uint32_t j = 0; j < nh; ++j) hs.h[j] = h[j];
    // ascending order
    for (uint32_t i = 1; i < nh; ++i)
        for (uint32_t j = i; j > 0 && hs.h[j - 1] > hs.h[j]; --j) {
            uint32_t t = hs.h[j];
            hs.h[j] = hs.h[j - 1];
            hs.h[j - 1] = t;
        }
    return hs;
}

}  // namespace

cudaError_t launch_apply_1q(float2* a, uint32_t n, uint32_t t, const Mat2f& m, cudaStream_t s) {
    const uint64_t dim = uint64_t{1} << n;
    if (t == 0) {
        const uint64_t items = dim / 2;
        k_u1_lo<<<sweep_grid(items, kThreads), kThreads, 0, s>>>(a, items, m);
    } else {
        const uint64_t items = dim / 4;
        k_u1_hi<<<sweep_grid(items, kThreads), kThreads, 0, s>>>(a, items, t, m);
    }
    return cudaGetLastError();
}

cudaError_t launch_apply_diag1(float2* a, uint32_t n, uint32_t t, float2 d0, float2 d1, cudaStream_t s) {
    const uint64_t dim = uint64_t{1} << n;
    const bool only_one = (t >= 1) && d0.x == 1.f && d0.y == 0.f;
    const uint64_t items = only_one ? dim / 4 : dim / 2;
    k_diag1<<<sweep_grid(items, kThreads), kThreads, 0, s>>>(a, items, t, d0, d1, only_one ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_swap_subspace(float2* a, uint32_t n, const uint32_t* holes, uint32_t nh, uint64_t ma,
                                 uint64_t mb, cudaStream_t s) {
    Holes hs = make_holes(holes, nh);
    const uint64_t iters = (uint64_t{1} << n) >> nh;
    if (hs.h[0] >= 1 && iters >= 2) {
        const uint64_t items = iters / 2;
        k_swap_subspace<true><<<sweep_grid(items, kThreads), kThreads, 0, s>>>(a, items, hs, ma, mb);
    } else {
        k_swap_subspace<false><<<sweep_grid(iters, kThreads), kThreads, 0, s>>>(a, iters, hs, ma, mb);
    }
    return cudaGetLastError();
}

cudaError_t launch_phase_mask(float2* a, uint32_t n, const uint32_t* holes, uint32_t nh, uint64_t mask, float2 ph,
                              cudaStream_t s) {
    Holes hs = make_holes(holes, nh);
    const uint64_t iters = (uint64_t{1} << n) >> nh;
    if (hs.h[0] >= 1 && iters >= 2) {
        const uint64_t items = iters / 2;
        k_phase_mask<true><<<sweep_grid(items, kThreads), kThreads, 0, s>>>(a, items, hs, mask, ph);
    } else {
        k_phase_mask<false><<<sweep_grid(iters, kThreads), kThreads, 0, s>>>(a, iters, hs, mask, ph);
    }
    return cudaGetLastError();
}

cudaError_t launch_apply_dense(float2* a, uint32_t n, const uint32_t* q, uint32_t k, const float2* mat,
                               cudaStream_t s) {
    Holes hs = make_holes(q, k);
    Offsets off{};
    for (uint32_t j = 0; j < (1u << k); ++j) {
        uint64_t o = 0;
        for (uint32_t b = 0; b < k; ++b)
            if ((j >> b) & 1u) o |= uint64_t{1} << q[b];
        off.o[j] = o;
    }
    const uint64_t groups = (uint64_t{1} << n) >> k;
    const unsigned grid = sweep_grid(groups, 128, 8);
    switch (k) {
    case 1: k_dense<1><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    case 2: k_dense<2><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    case 3: k_dense<3><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    case 4: k_dense<4><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    case 5: k_dense<5><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    case 6: k_dense<6><<<grid, 128, 0, s>>>(a, groups, hs, off, mat); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace qlb

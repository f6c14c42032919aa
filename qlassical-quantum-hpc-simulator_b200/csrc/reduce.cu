// reduce.cu -- FP64 reductions over the complex64 state, measurement
// collapse and counter-based sampling.
//
//   norm_sq       sum |a|^2 (the check inside initialize(span),
//                 cpu_state_vector.hpp:97-106)
//   prob_one      P(qubit = 1) (apply_measure, cpu_openmp_engine.hpp:622-630)
//   marginals     P(q = 1) for every qubit in ONE sweep -> <Z_q> = 1 - 2 P1
//   collapse      zero one half, rescale the other (:649-670)
//   sample        shots from |a|^2 via per-chunk FP64 sums + a scan; the
//                 uniform draws come from SplitMix64 (Steele, Lea & Flood,
//                 2014) keyed by (seed, shot), so a shot's value does not
//                 depend on which other requests share the launch.
// Every accumulation is in double; each thread adds complex64 inputs
// widened to double.
#include "common.cuh"
#include "kernels.h"

namespace qlb {

namespace {
constexpr unsigned kThreads = 256;
constexpr uint32_t kMaxQubits = 34;
constexpr uint32_t kChunkLog2 = 13;   // marginals: 2^13 amplitudes per block iteration

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; every thread gets the result. `sh` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double p2(float2 v) {
    return static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
}

__global__ void __launch_bounds__(kThreads) k_norm_partial(const float2* __restrict__ a, uint64_t dim,
                                                           double* __restrict__ partial) {
    __shared__ double sh[32];
    double acc = 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t n4 = dim / 2;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < n4; k += stride) {
        float4 x = reinterpret_cast<const float4*>(a)[k];
        acc += p2(make_float2(x.x, x.y)) + p2(make_float2(x.z, x.w));
    }
    if (dim == 1 && blockIdx.x == 0 && threadIdx.x == 0) acc = p2(a[0]);
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kThreads) k_prob_one_partial(const float2* __restrict__ a, uint64_t dim,
                                                               uint32_t q, double* __restrict__ partial) {
    __shared__ double sh[32];
    double acc = 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    if (q == 0) {
        const uint64_t n4 = dim / 2;
        for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < n4; k += stride) {
            float4 x = reinterpret_cast<const float4*>(a)[k];
            acc += p2(make_float2(x.z, x.w));
        }
    } else {
        const uint64_t items = dim / 4;
        for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
            const uint64_t i1 = insert_zero_bit(2 * k, q) | (uint64_t{1} << q);
            float4 x = *reinterpret_cast<const float4*>(a + i1);
            acc += p2(make_float2(x.x, x.y)) + p2(make_float2(x.z, x.w));
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Sums `count` vectors of length `width` laid out as partial[b * width + i].
__global__ void k_finalize(const double* __restrict__ partial, uint32_t count, uint32_t width,
                           double* __restrict__ out) {
    __shared__ double sh[32];
    for (uint32_t i = 0; i < width; ++i) {
        double acc = 0.0;
        for (uint32_t b = threadIdx.x; b < count; b += blockDim.x) acc += partial[static_cast<uint64_t>(b) * width + i];
        acc = block_sum(acc, sh);
        if (threadIdx.x == 0) out[i] = acc;
    }
}

// Small states (n < 13): one block, plain per-amplitude loop.
__global__ void k_marginals_small(const float2* __restrict__ a, uint32_t n, double* __restrict__ out) {
    __shared__ double sh[32];
    const uint64_t dim = uint64_t{1} << n;
    double tot = 0.0, acc[kChunkLog2];
#pragma unroll
    for (uint32_t q = 0; q < kChunkLog2; ++q) acc[q] = 0.0;
    for (uint64_t i = threadIdx.x; i < dim; i += blockDim.x) {
        const double p = p2(a[i]);
        tot += p;
#pragma unroll
        for (uint32_t q = 0; q < kChunkLog2; ++q)
            if (q < n && ((i >> q) & 1)) acc[q] += p;
    }
    tot = block_sum(tot, sh);
    if (threadIdx.x == 0) out[0] = tot;
#pragma unroll
    for (uint32_t q = 0; q < kChunkLog2; ++q) {
        double v = block_sum(acc[q], sh);
        if (q < n && threadIdx.x == 0) out[1 + q] = v;
    }
}

// n >= 13: each block iterates chunks of 2^13 amplitudes; inside a chunk,
// float4 j*256+tid holds amplitudes with bit 0 = lane of the float4,
// bits 1..8 = tid, bits 9..12 = j, bits >= 13 = chunk index.
__global__ void __launch_bounds__(kThreads) k_marginals(const float2* __restrict__ a, uint32_t n,
                                                        double* __restrict__ partial) {
    __shared__ double sh[32];
    const uint64_t chunks = uint64_t{1} << (n - kChunkLog2);
    double tot = 0.0, b0 = 0.0, jb[4] = {0.0, 0.0, 0.0, 0.0}, hi[kMaxQubits - kChunkLog2];
#pragma unroll
    for (uint32_t q = 0; q < kMaxQubits - kChunkLog2; ++q) hi[q] = 0.0;
    const float4* a4 = reinterpret_cast<const float4*>(a);
    for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        double csum = 0.0;
#pragma unroll 4
        for (uint32_t j = 0; j < 16; ++j) {
            float4 x = a4[(c << (kChunkLog2 - 1)) + j * kThreads + threadIdx.x];
            const double pe = p2(make_float2(x.x, x.y)), po = p2(make_float2(x.z, x.w));
            const double s = pe + po;
            b0 += po;
            csum += s;
#pragma unroll
            for (uint32_t jj = 0; jj < 4; ++jj)
                if ((j >> jj) & 1) jb[jj] += s;
        }
        tot += csum;
#pragma unroll
        for (uint32_t q = 0; q < kMaxQubits - kChunkLog2; ++q)
            if (q + kChunkLog2 < n && ((c >> q) & 1)) hi[q] += csum;
    }
    double* out = partial + static_cast<uint64_t>(blockIdx.x) * (n + 1);
    double v = block_sum(tot, sh);
    if (threadIdx.x == 0) out[0] = v;
    v = block_sum(b0, sh);
    if (threadIdx.x == 0) out[1] = v;
#pragma unroll
    for (uint32_t q = 1; q <= 8; ++q) {
        v = block_sum(((threadIdx.x >> (q - 1)) & 1) ? tot : 0.0, sh);
        if (threadIdx.x == 0) out[1 + q] = v;
    }
#pragma unroll
    for (uint32_t jj = 0; jj < 4; ++jj) {
        v = block_sum(jb[jj], sh);
        if (threadIdx.x == 0) out[1 + 9 + jj] = v;
    }
#pragma unroll
    for (uint32_t q = 0; q < kMaxQubits - kChunkLog2; ++q) {
        if (q + kChunkLog2 < n) {
            v = block_sum(hi[q], sh);
            if (threadIdx.x == 0) out[1 + kChunkLog2 + q] = v;
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_collapse(float2* __restrict__ a, uint64_t dim, uint32_t t,
                                                       int outcome, float scale) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t half = dim / 2;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < half; k += stride) {
        const uint64_t i0 = insert_zero_bit(k, t), i1 = i0 | (uint64_t{1} << t);
        const uint64_t keep = outcome ? i1 : i0, drop = outcome ? i0 : i1;
        float2 v = a[keep];
        a[keep] = make_float2(v.x * scale, v.y * scale);
        a[drop] = make_float2(0.f, 0.f);
    }
}

// ---- sampling -------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) k_chunk_sums(const float2* __restrict__ a, uint32_t chunk_log2,
                                                         uint64_t chunks, double* __restrict__ sums) {
    __shared__ double sh[32];
    const uint64_t len = uint64_t{1} << chunk_log2;
    for (uint64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        double acc = 0.0;
        for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) acc += p2(a[c * len + i]);
        acc = block_sum(acc, sh);
        if (threadIdx.x == 0) sums[c] = acc;
    }
}

// In-place inclusive scan of m doubles by one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan(double* __restrict__ v, uint64_t m) {
    __shared__ double tot[1024];
    const uint64_t seg = (m + blockDim.x - 1) / blockDim.x;
    const uint64_t b = threadIdx.x * seg, e = (b + seg < m) ? b + seg : m;
    double run = 0.0;
    for (uint64_t i = b; i < e; ++i) { run += v[i]; v[i] = run; }
    tot[threadIdx.x] = run;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (unsigned t = 0; t < blockDim.x; ++t) { double x = tot[t]; tot[t] = r; r += x; }
    }
    __syncthreads();
    const double off = tot[threadIdx.x];
    for (uint64_t i = b; i < e; ++i) v[i] += off;
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

// One warp per shot: binary search over the chunk CDF, then a warp scan
// inside the chunk.
__global__ void __launch_bounds__(kThreads) k_sample(const float2* __restrict__ a, uint32_t chunk_log2,
                                                     uint64_t chunks, const double* __restrict__ cdf,
                                                     uint64_t seed, uint64_t shots, uint64_t* __restrict__ out) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t warps = static_cast<uint64_t>(gridDim.x) * (blockDim.x >> 5);
    const uint64_t len = uint64_t{1} << chunk_log2;
    const double total = cdf[chunks - 1];
    for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x >> 5) + (threadIdx.x >> 5); s < shots;
         s += warps) {
        const uint64_t r = splitmix64(seed ^ splitmix64(s));
        const double u = static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0) * total;
        uint64_t lo = 0, hi = chunks - 1;  // first c with cdf[c] > u
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (cdf[mid] > u) hi = mid; else lo = mid + 1;
        }
        const uint64_t c = lo;
        double target = u - (c ? cdf[c - 1] : 0.0);
        uint64_t found = ~uint64_t{0}, last_nz = c * len;
        for (uint64_t base = 0; base < len && found == ~uint64_t{0}; base += 32) {
            const uint64_t i = c * len + base + lane;
            const double p = (base + lane < len) ? p2(a[i]) : 0.0;
            double incl = p;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                double y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= static_cast<unsigned>(o)) incl += y;
            }
            const unsigned hit = __ballot_sync(0xffffffffu, incl > target && p > 0.0);
            const unsigned nz = __ballot_sync(0xffffffffu, p > 0.0);
            if (nz) last_nz = c * len + base + (31 - __clz(nz));
            if (hit) {
                found = c * len + base + (__ffs(hit) - 1);
            } else {
                target -= __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        if (lane == 0) out[s] = (found != ~uint64_t{0}) ? found : last_nz;
    }
}

}  // namespace

static unsigned reduce_grid(uint64_t items) { return sweep_grid(items, kThreads, 4); }

cudaError_t launch_norm_sq(const float2* a, uint64_t dim, double* partial, uint32_t partial_cap, double* out,
                           cudaStream_t s) {
    unsigned g = reduce_grid(dim / 2 > 0 ? dim / 2 : 1);
    if (g > partial_cap) g = partial_cap;
    k_norm_partial<<<g, kThreads, 0, s>>>(a, dim, partial);
    k_finalize<<<1, kThreads, 0, s>>>(partial, g, 1, out);
    return cudaGetLastError();
}

cudaError_t launch_prob_one(const float2* a, uint32_t n, uint32_t qubit, double* partial, uint32_t partial_cap,
                            double* out, cudaStream_t s) {
    const uint64_t dim = uint64_t{1} << n;
    if (n == 0) return cudaErrorInvalidValue;
    if (n == 1) {  // dim == 2: one float4, q == 0
        k_prob_one_partial<<<1, kThreads, 0, s>>>(a, dim, 0, partial);
        k_finalize<<<1, kThreads, 0, s>>>(partial, 1, 1, out);
        return cudaGetLastError();
    }
    unsigned g = reduce_grid(dim / 4);
    if (g > partial_cap) g = partial_cap;
    k_prob_one_partial<<<g, kThreads, 0, s>>>(a, dim, qubit, partial);
    k_finalize<<<1, kThreads, 0, s>>>(partial, g, 1, out);
    return cudaGetLastError();
}

uint32_t marginals_partial_size(uint32_t n) {
    return static_cast<uint32_t>(sm_count()) * 4u * (n + 1);
}

cudaError_t launch_qubit_marginals(const float2* a, uint32_t n, double* partial, uint32_t partial_cap,
                                   double* out, cudaStream_t s) {
    if (n > kMaxQubits) return cudaErrorInvalidValue;
    if (n < kChunkLog2) {
        k_marginals_small<<<1, kThreads, 0, s>>>(a, n, out);
        return cudaGetLastError();
    }
    const uint64_t chunks = uint64_t{1} << (n - kChunkLog2);
    uint64_t g = static_cast<uint64_t>(sm_count()) * 4u;
    if (g > chunks) g = chunks;
    if (g * (n + 1) > partial_cap) g = partial_cap / (n + 1);
    if (g == 0) return cudaErrorInvalidValue;
    k_marginals<<<static_cast<unsigned>(g), kThreads, 0, s>>>(a, n, partial);
    k_finalize<<<1, kThreads, 0, s>>>(partial, static_cast<uint32_t>(g), n + 1, out);
    return cudaGetLastError();
}

cudaError_t launch_collapse(float2* a, uint32_t n, uint32_t t, int outcome, float scale, cudaStream_t s) {
    const uint64_t dim = uint64_t{1} << n;
    k_collapse<<<sweep_grid(dim / 2, kThreads), kThreads, 0, s>>>(a, dim, t, outcome, scale);
    return cudaGetLastError();
}

uint64_t sample_scratch_doubles(uint32_t n) {
    return n > kSampleChunkLog2 ? (uint64_t{1} << (n - kSampleChunkLog2)) : 1;
}

cudaError_t launch_sample(const float2* a, uint32_t n, uint64_t seed, uint64_t shots, double* chunk_sums,
                          uint64_t* out, cudaStream_t s) {
    const uint32_t cl = n < kSampleChunkLog2 ? n : kSampleChunkLog2;
    const uint64_t chunks = uint64_t{1} << (n - cl);
    k_chunk_sums<<<reduce_grid(chunks * kThreads), kThreads, 0, s>>>(a, cl, chunks, chunk_sums);
    k_scan<<<1, 1024, 0, s>>>(chunk_sums, chunks);
    if (shots) {
        const uint64_t warps_needed = shots;
        unsigned g = static_cast<unsigned>((warps_needed + 7) / 8);
        const unsigned cap = static_cast<unsigned>(sm_count()) * 8u;
        if (g > cap) g = cap;
        k_sample<<<g, kThreads, 0, s>>>(a, cl, chunks, chunk_sums, seed, shots, out);
    }
    return cudaGetLastError();
}

}  // namespace qlb

// check64.cu -- the FP64 checker: a complex128 state vector on the device
// that executes a program gate by gate in double precision.
//
// It is the GPU-resident counterpart of the reference engine's own
// arithmetic (complex128 throughout, cpu_openmp_engine.hpp:143-225) and
// exists to measure the complex64 engine's error at sizes where a host
// complex128 run is too slow: the same program runs here and through the
// engine, and qlb_check64_compare() reduces max |delta amplitude| and the
// infidelity 1 - |<ref|psi>|^2 / (<ref|ref><psi|psi>) over the whole state
// in FP64.  Gate matrices are built in double from the float parameter, as
// the reference kernels do (:408-465), and never rounded to float.
// GLOBAL_SWAP exchanges two physical qubits (the intended semantics; the
// reference's no-op at :217-219 is a bug): the checker keeps a
// physical->memory qubit map instead of moving data, so the state stays in
// logical order, as the engine's does.
//
// Kernels are HBM-bound sweeps (32 B per touched amplitude); one launch per
// instruction.  MEASURE is not supported (the checker has no RNG).
#include "abi.h"

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "tile.h"

struct qlb_check64 {
    double2* d = nullptr;
    uint32_t n = 0;
    cudaStream_t stream = nullptr;
    qlb::DeviceBuffer mats, partial;
    qlb::PinnedBuffer host;
};

namespace qlb {
namespace {

constexpr unsigned kT = 256;
constexpr uint32_t kCmpBlocksPerSm = 4;

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__global__ void k64_init(double2* __restrict__ a, uint64_t dim) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < dim; i += stride)
        a[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
}

// Dense 2^K x 2^K complex128 matrix (row-major, matrix bit j <-> offset bit
// off.o[1 << j]) on every group of 2^K amplitudes.
struct Offsets64 {
    uint64_t o[64];
};
template <int K>
__global__ void __launch_bounds__(128) k64_dense(double2* __restrict__ a, uint64_t groups, Holes hs, Offsets64 off,
                                                 const double2* __restrict__ mat) {
    constexpr int D = 1 << K;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g < groups; g += stride) {
        const uint64_t base = insert_zero_bits(g, hs);
        double2 v[D];
#pragma unroll
        for (int j = 0; j < D; ++j) v[j] = a[base | off.o[j]];
#pragma unroll 1
        for (int r = 0; r < D; ++r) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const double2 m = __ldg(mat + r * D + c);   // warp-uniform: a broadcast
                acc.x = fma(m.x, v[c].x, acc.x);
                acc.x = fma(-m.y, v[c].y, acc.x);
                acc.y = fma(m.x, v[c].y, acc.y);
                acc.y = fma(m.y, v[c].x, acc.y);
            }
            a[base | off.o[r]] = acc;
        }
    }
}

// a[base | ma] <-> a[base | mb] over the bases with zeros at the holes.
__global__ void k64_swap(double2* __restrict__ a, uint64_t items, Holes hs, uint64_t ma, uint64_t mb) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        const uint64_t base = insert_zero_bits(k, hs);
        const double2 x = a[base | ma], y = a[base | mb];
        a[base | ma] = y;
        a[base | mb] = x;
    }
}

// a[i] *= ph for every i with all bits of `mask` set.
__global__ void k64_phase(double2* __restrict__ a, uint64_t items, Holes hs, uint64_t mask, double2 ph) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < items; k += stride) {
        const uint64_t i = insert_zero_bits(k, hs) | mask;
        a[i] = zmul(ph, a[i]);
    }
}

// Per block: sum conj(r) p (2 doubles), sum |r|^2, sum |p|^2, max |r - p|.
__global__ void __launch_bounds__(kT) k64_compare(const double2* __restrict__ r, const float2* __restrict__ p,
                                                  uint64_t dim, double* __restrict__ partial) {
    double ore = 0.0, oim = 0.0, nr = 0.0, np = 0.0, mx = 0.0;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < dim; i += stride) {
        const double2 a = r[i];
        const float2 bf = p[i];
        const double bx = bf.x, by = bf.y;
        ore = fma(a.x, bx, fma(a.y, by, ore));
        oim = fma(a.x, by, fma(-a.y, bx, oim));
        nr = fma(a.x, a.x, fma(a.y, a.y, nr));
        np = fma(bx, bx, fma(by, by, np));
        const double dx = a.x - bx, dy = a.y - by;
        mx = fmax(mx, sqrt(dx * dx + dy * dy));
    }
    __shared__ double s[5][kT / 32];
    double v[5] = {ore, oim, nr, np, mx};
#pragma unroll
    for (int j = 0; j < 5; ++j)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_xor_sync(0xFFFFFFFFu, v[j], o);
            v[j] = (j == 4) ? fmax(v[j], w) : v[j] + w;
        }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int j = 0; j < 5; ++j) s[j][w] = v[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[5] = {0, 0, 0, 0, 0};
        for (int k = 0; k < kT / 32; ++k)
            for (int j = 0; j < 5; ++j) t[j] = (j == 4) ? fmax(t[j], s[j][k]) : t[j] + s[j][k];
        for (int j = 0; j < 5; ++j) partial[5 * blockIdx.x + j] = t[j];
    }
}

using Mat64 = std::vector<double2>;

// The 2x2 of a 1-qubit gate in double from the float parameter
// (cpu_openmp_engine.hpp:337-465).
Mat64 matrix_1q(uint8_t type, float param) {
    const double r2 = 1.0 / std::sqrt(2.0);
    const double h = static_cast<double>(param) * 0.5, c = std::cos(h), s = std::sin(h);
    switch (type) {
    case QLB_H: return {{r2, 0}, {r2, 0}, {r2, 0}, {-r2, 0}};
    case QLB_Y: return {{0, 0}, {0, -1}, {0, 1}, {0, 0}};
    case QLB_RX: return {{c, 0}, {0, -s}, {0, -s}, {c, 0}};
    case QLB_RY: return {{c, 0}, {-s, 0}, {s, 0}, {c, 0}};
    case QLB_RZ: return {{std::cos(-h), std::sin(-h)}, {0, 0}, {0, 0}, {std::cos(h), std::sin(h)}};
    default: return {{1, 0}, {0, 0}, {0, 0}, {1, 0}};
    }
}

Holes holes_of(const uint32_t* q, uint32_t k) {
    Holes hs{};
    hs.n = k;
    for (uint32_t j = 0; j < k; ++j) hs.h[j] = q[j];
    for (uint32_t i = 1; i < k; ++i)
        for (uint32_t j = i; j > 0 && hs.h[j - 1] > hs.h[j]; --j) std::swap(hs.h[j], hs.h[j - 1]);
    return hs;
}

void launch_dense64(qlb_check64& c, const uint32_t* q, uint32_t k, const double2* dmat) {
    const Holes hs = holes_of(q, k);
    Offsets64 off{};
    for (uint32_t j = 0; j < (1u << k); ++j) {
        uint64_t o = 0;
        for (uint32_t b = 0; b < k; ++b)
            if ((j >> b) & 1u) o |= uint64_t{1} << q[b];
        off.o[j] = o;
    }
    const uint64_t groups = (uint64_t{1} << c.n) >> k;
    const unsigned grid = sweep_grid(groups, 128, 8);
    switch (k) {
    case 1: k64_dense<1><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    case 2: k64_dense<2><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    case 3: k64_dense<3><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    case 4: k64_dense<4><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    case 5: k64_dense<5><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    case 6: k64_dense<6><<<grid, 128, 0, c.stream>>>(c.d, groups, hs, off, dmat); break;
    default: fail(QLB_ERR_INVALID_ARG, "dense arity must be 1..6");
    }
    check_cuda(cudaGetLastError(), "check64 dense");
}

void launch_swap64(qlb_check64& c, const uint32_t* q, uint32_t k, uint64_t ma, uint64_t mb) {
    const Holes hs = holes_of(q, k);
    const uint64_t items = (uint64_t{1} << c.n) >> k;
    k64_swap<<<sweep_grid(items, kT), kT, 0, c.stream>>>(c.d, items, hs, ma, mb);
    check_cuda(cudaGetLastError(), "check64 swap");
}

void launch_phase64(qlb_check64& c, const uint32_t* q, uint32_t k, double2 ph) {
    const Holes hs = holes_of(q, k);
    uint64_t mask = 0;
    for (uint32_t j = 0; j < k; ++j) mask |= uint64_t{1} << q[j];
    const uint64_t items = (uint64_t{1} << c.n) >> k;
    k64_phase<<<sweep_grid(items, kT), kT, 0, c.stream>>>(c.d, items, hs, mask, ph);
    check_cuda(cudaGetLastError(), "check64 phase");
}

void execute64(qlb_check64& c, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool) {
    // Validate everything and collect the dense matrices first (one upload).
    std::vector<double2> host;
    std::vector<uint64_t> where(count, 0);
    for (uint64_t g = 0; g < count; ++g) {
        const qlb_gate_instr& in = prog[g];
        const uint32_t k = validate_instr(in, c.n, pool);
        if (in.type == QLB_MEASURE) fail(QLB_ERR_INVALID_ARG, "the FP64 checker does not execute MEASURE");
        where[g] = host.size();
        if (in.type == QLB_H || in.type == QLB_Y || in.type == QLB_RX || in.type == QLB_RY || in.type == QLB_RZ) {
            const Mat64 m = matrix_1q(in.type, in.payload.param);
            host.insert(host.end(), m.begin(), m.end());
        } else if (in.type == QLB_UNITARY || in.type == QLB_FUSED_BLOCK) {
            const qlb_matrix_entry& e = pool->metadata[in.payload.matrix_idx];
            const double* src = pool->data + 2 * static_cast<uint64_t>(e.offset);
            for (uint32_t i = 0; i < (1u << (2 * k)); ++i) host.push_back(make_double2(src[2 * i], src[2 * i + 1]));
        }
    }
    double2* dm = nullptr;
    if (!host.empty()) {
        dm = static_cast<double2*>(c.mats.ensure(host.size() * sizeof(double2)));
        check_cuda(cudaMemcpyAsync(dm, host.data(), host.size() * sizeof(double2), cudaMemcpyHostToDevice, c.stream),
                   "check64 matrices");
    }
    uint32_t mem[64];
    for (uint32_t i = 0; i < 64; ++i) mem[i] = i;
    for (uint64_t g = 0; g < count; ++g) {
        const qlb_gate_instr& in = prog[g];
        uint32_t q[6] = {0, 0, 0, 0, 0, 0};
        const uint32_t k = (in.type == QLB_UNITARY || in.type == QLB_FUSED_BLOCK) ? (in.flags_arity & 0x0Fu)
                           : (in.type == QLB_CCX || in.type == QLB_CSWAP)                ? 3u
                           : (in.type == QLB_CX || in.type == QLB_SWAP || in.type == QLB_CZ || in.type == QLB_CP ||
                              in.type == QLB_GLOBAL_SWAP)                                 ? 2u
                           : (in.type == QLB_BARRIER)                                     ? 0u
                                                                                          : 1u;
        for (uint32_t j = 0; j < k; ++j) q[j] = mem[instr_qubit(in, j)];
        auto bit = [](uint32_t x) { return uint64_t{1} << x; };
        switch (in.type) {
        case QLB_H: case QLB_Y: case QLB_RX: case QLB_RY: case QLB_RZ:
        case QLB_UNITARY: case QLB_FUSED_BLOCK:
            launch_dense64(c, q, k, dm + where[g]);
            break;
        case QLB_X: launch_swap64(c, q, 1, 0, bit(q[0])); break;
        case QLB_Z: launch_phase64(c, q, 1, make_double2(-1.0, 0.0)); break;
        case QLB_S: launch_phase64(c, q, 1, make_double2(0.0, 1.0)); break;
        case QLB_CX: launch_swap64(c, q, 2, bit(q[0]), bit(q[0]) | bit(q[1])); break;
        case QLB_SWAP: launch_swap64(c, q, 2, bit(q[1]), bit(q[0])); break;
        case QLB_CZ: launch_phase64(c, q, 2, make_double2(-1.0, 0.0)); break;
        case QLB_CP: {
            const double phi = static_cast<double>(in.payload.param);
            launch_phase64(c, q, 2, make_double2(std::cos(phi), std::sin(phi)));
            break;
        }
        case QLB_CCX: launch_swap64(c, q, 3, bit(q[0]) | bit(q[1]), bit(q[0]) | bit(q[1]) | bit(q[2])); break;
        case QLB_CSWAP: launch_swap64(c, q, 3, bit(q[0]) | bit(q[2]), bit(q[0]) | bit(q[1])); break;
        case QLB_GLOBAL_SWAP: std::swap(mem[in.qubits[0]], mem[in.qubits[1]]); break;
        default: break;   // BARRIER
        }
    }
    // No restore is needed: memory bit mem[p] holds what physical bit p
    // would hold after eager swaps, and mem[] equals the eager
    // physical->logical map, so memory bit b holds logical qubit b.
    check_cuda(cudaStreamSynchronize(c.stream), "check64 execute");
}

}  // namespace
}  // namespace qlb

using namespace qlb;

extern "C" {

int qlb_check64_create(qlb_check64_t* out, uint32_t num_qubits) {
    return guarded([&] {
        need(out, "out");
        if (num_qubits < 1 || num_qubits > 33) fail(QLB_ERR_INVALID_ARG, "FP64 checker: 1..33 qubits");
        auto* c = new qlb_check64();
        try {
            check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            const uint64_t dim = uint64_t{1} << num_qubits;
            void* p = nullptr;
            check_cuda(cudaMalloc(&p, dim * sizeof(double2)), "cudaMalloc(FP64 state)");
            c->d = static_cast<double2*>(p);
            c->n = num_qubits;
            k64_init<<<sweep_grid(dim, kT), kT, 0, c->stream>>>(c->d, dim);
            check_cuda(cudaGetLastError(), "check64 init");
            check_cuda(cudaStreamSynchronize(c->stream), "check64 init sync");
        } catch (...) {
            if (c->d) cudaFree(c->d);
            if (c->stream) cudaStreamDestroy(c->stream);
            delete c;
            throw;
        }
        *out = c;
    });
}

int qlb_check64_destroy(qlb_check64_t c) {
    return guarded([&] {
        if (!c) return;
        if (c->stream) cudaStreamSynchronize(c->stream);
        if (c->d) cudaFree(c->d);
        c->mats.release();
        c->partial.release();
        c->host.release();
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
    });
}

int qlb_check64_execute(qlb_check64_t c, const qlb_gate_instr* program, uint64_t count, const qlb_pool_view* pool) {
    return guarded([&] {
        need(c, "checker");
        if (count) need(program, "program");
        execute64(*c, program, count, pool);
    });
}

int qlb_check64_compare(qlb_check64_t c, const void* state_float2, qlb_check64_result* out) {
    return guarded([&] {
        need(c, "checker");
        need(state_float2, "state");
        need(out, "out");
        const uint64_t dim = uint64_t{1} << c->n;
        const uint32_t blocks = static_cast<uint32_t>(sm_count()) * kCmpBlocksPerSm;
        double* part = static_cast<double*>(c->partial.ensure(blocks * 5 * sizeof(double)));
        k64_compare<<<blocks, kT, 0, c->stream>>>(c->d, static_cast<const float2*>(state_float2), dim, part);
        check_cuda(cudaGetLastError(), "check64 compare");
        double* h = static_cast<double*>(c->host.ensure(blocks * 5 * sizeof(double)));
        check_cuda(cudaMemcpyAsync(h, part, blocks * 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                   "check64 D2H");
        check_cuda(cudaStreamSynchronize(c->stream), "check64 compare sync");
        double ore = 0, oim = 0, nr = 0, np = 0, mx = 0;
        for (uint32_t b = 0; b < blocks; ++b) {
            ore += h[5 * b];
            oim += h[5 * b + 1];
            nr += h[5 * b + 2];
            np += h[5 * b + 3];
            mx = std::fmax(mx, h[5 * b + 4]);
        }
        out->max_abs_diff = mx;
        out->norm_ref = nr;
        out->norm_state = np;
        out->overlap_re = ore;
        out->overlap_im = oim;
        out->infidelity = 1.0 - (ore * ore + oim * oim) / (nr * np);
    });
}

int qlb_check64_download(qlb_check64_t c, double* out_c128, uint64_t dim) {
    return guarded([&] {
        need(c, "checker");
        need(out_c128, "out");
        if (dim != (uint64_t{1} << c->n)) fail(QLB_ERR_INVALID_ARG, "output size does not match the state dimension");
        check_cuda(cudaMemcpyAsync(out_c128, c->d, dim * sizeof(double2), cudaMemcpyDeviceToHost, c->stream),
                   "check64 download");
        check_cuda(cudaStreamSynchronize(c->stream), "check64 download sync");
    });
}

}  // extern "C"

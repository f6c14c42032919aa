// noalloc.cu -- <Z_q> for every qubit without allocating any memory.
//
// Who needs this: code that must not allocate device memory while it runs --
// above all a continuous-batching serving loop, which admits requests by
// accounting every byte of free HBM to the state vectors it keeps resident.
// A reduction that called cudaMalloc for its scratch would take memory the
// admission control never saw, and cudaMalloc / cudaFree synchronize the
// device, stalling the kernels of every other request in flight.  This entry
// point uses a fixed scratch array that lives in the library's own device
// image instead, so the only memory it touches besides the caller's state
// and output is that array.
//
// Limits and rules (also stated in include/qlassical_b200.h):
//   - the scratch holds kNoAllocScratchDoubles doubles (about 176 KiB) on
//     every GPU where the entry point has been called, from its first call
//     (the library's modules load lazily, so the array is committed when the
//     first call looks up its address) until the library is unloaded: a
//     caller that budgets free memory makes a warm-up call first;
//   - states of 1..34 qubits are accepted, anything else is rejected;
//   - all calls share the one array, so two calls whose kernels overlap on
//     the GPU (different streams, or host threads) race and corrupt each
//     other's result; serialize them;
//   - the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.  The address is cached for the life
//     of the process: after a cudaDeviceReset of that device it is stale, so
//     a process that resets a device must not call this entry point again;
//   - nothing in the scratch needs to start at zero: every partial slot the
//     reduction reads is written by the same call first.
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/qlassical_b200.h"
#include "common.cuh"
#include "engine.h"
#include "kernels.h"

namespace qlb {
namespace {

constexpr uint32_t kNoAllocMaxQubits = 34;
// partial sums: up to 4 CTAs per SM on up to 160 SMs, (n + 1) doubles each,
// plus (n + 1) doubles for the final sums
constexpr size_t kNoAllocPartialDoubles = size_t{4} * 160 * (kNoAllocMaxQubits + 1);
constexpr size_t kNoAllocScratchDoubles = kNoAllocPartialDoubles + 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device, with that device current).
double* scratch_address() {
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) fail(QLB_ERR_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            fail(QLB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    return static_cast<double*>(g_noalloc_addr[dev]);
}

}  // namespace
}  // namespace qlb

extern "C" int qlb_expect_z_noalloc(const void* state_float2, uint32_t num_qubits, double* out,
                                    void* cuda_stream) {
    using namespace qlb;
    try {
        if (!state_float2 || !out) fail(QLB_ERR_INVALID_ARG, "qlb_expect_z_noalloc: state and out must be non-null");
        if (num_qubits < 1 || num_qubits > kNoAllocMaxQubits)
            fail(QLB_ERR_INVALID_ARG, "qlb_expect_z_noalloc: num_qubits must be 1..34 (fixed scratch size)");
        cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
        double* scratch = scratch_address();
        double* partial = scratch;
        double* sums = scratch + kNoAllocPartialDoubles;
        check_cuda(launch_qubit_marginals(static_cast<const float2*>(state_float2), num_qubits, partial,
                                          static_cast<uint32_t>(kNoAllocPartialDoubles), sums, s),
                   "no-alloc marginals");
        double host[kNoAllocMaxQubits + 1];
        check_cuda(cudaMemcpyAsync(host, sums, (num_qubits + 1) * sizeof(double), cudaMemcpyDeviceToHost, s),
                   "no-alloc D2H");
        check_cuda(cudaStreamSynchronize(s), "no-alloc sync");
        for (uint32_t q = 0; q < num_qubits; ++q) out[q] = host[0] - 2.0 * host[1 + q];
        return QLB_OK;
    } catch (const Error& err) {
        set_last_error(err.msg);
        return err.code;
    } catch (...) {
        set_last_error("qlb_expect_z_noalloc: unexpected failure");
        return QLB_ERR_CUDA;
    }
}

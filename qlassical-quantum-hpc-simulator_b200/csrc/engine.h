// engine.h -- C++ engine objects behind the C ABI (qlassical_b200.h).
#pragma once

#include <array>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qlassical_b200.h"
#include "tile.h"

struct qlb_state {
    float2* d = nullptr;   // 2^n complex64 amplitudes (cudaMalloc, 256-B aligned)
    uint32_t n = 0;
    uint64_t dim = 0;      // 0 <=> empty
};

namespace qlb {

// Error carrier used inside the library; converted to a status at the ABI.
struct Error {
    qlb_status code;
    std::string msg;
};

[[noreturn]] void fail(qlb_status code, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
void set_last_error(const std::string& msg);

// Grow-only device / pinned host buffers.
struct DeviceBuffer {
    void* p = nullptr;
    size_t cap = 0;
    void* ensure(size_t bytes);
    void release();
    ~DeviceBuffer() { release(); }
};
struct PinnedBuffer {
    void* p = nullptr;
    size_t cap = 0;
    void* ensure(size_t bytes);
    void release();
    ~PinnedBuffer() { release(); }
};

void state_allocate(qlb_state& sv, uint32_t n);   // throws OOM
void state_free(qlb_state& sv);
// Uploads complex128 host amplitudes into sv (allocated), via device staging.
void state_upload_c128(qlb_state& sv, const double* amps, uint64_t dim, cudaStream_t s, DeviceBuffer& staging);
void state_download_c128(const qlb_state& sv, double* out, cudaStream_t s, DeviceBuffer& staging);

// Validates one instruction against the state size and pool; returns its
// arity (throws QLB_ERR_UNKNOWN_GATE / QLB_ERR_INVALID_ARG).
uint32_t validate_instr(const qlb_gate_instr& in, uint32_t n, const qlb_pool_view* pool);

struct TilePlanner;  // tile.cpp

}  // namespace qlb

struct qlb_engine {
    qlb_state sv;
    cudaStream_t stream = nullptr;
    std::mt19937_64 rng;                                  // cpu_openmp_engine.hpp:252
    std::uniform_real_distribution<double> dist{0.0, 1.0};  // :253
    std::vector<uint8_t> measurements;
    int mode = QLB_MODE_TILED;
    int physical_global_swap = 0;   // execute GLOBAL_SWAP as a data permutation
    double tc_min_cost = 10.0;      // TILED_TC: smallest fused-run cost sent to the tensor cores
    int tc_chain = 1;               // TILED_TC: chain kernel for passes of tensor-core ops only
    int tile_low = qlb::kTileLow;   // tiled modes: memory qubits 0..tile_low-1 in every tile
    qlb::DeviceBuffer red_partial, red_out, staging, err_flag, exec_plan;   // exec_plan: execute()'s plan image   // err_flag: device int set by bounded waits
    qlb::PinnedBuffer host_pinned, host_prog;
    qlb_exec_stats stats{};
    std::vector<double> last_marginals;
};

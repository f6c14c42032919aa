// engine.cpp -- CUDAStateVector / CUDAEngine behind the C ABI.
//
// The dispatch loop is the sm_100a counterpart of CPUOpenMPEngine::execute
// (cpu_openmp_engine.hpp:143-225): every reference instruction type is
// accepted, with the same error behaviour (unknown type -> QLB_ERR_UNKNOWN_GATE,
// which the C++ wrapper raises as std::runtime_error).  Gate matrices are
// built on the host in double from the float parameter, exactly as the
// reference kernels do (:408-465), and rounded once to complex64.
//
// GLOBAL_SWAP is executed as a qubit permutation (the reference's no-op at
// :217-219 is a bug): by default the permutation is applied lazily -- the
// engine keeps a physical->memory qubit map, so later instructions address
// the permuted qubits and the state stays in logical order in HBM, which is
// the same result as physically swapping and un-permuting at read-out.
// With the physical option it moves the data (a swap kernel, one
// bandwidth-bound pass) and restores logical order when execute() returns.
#include "abi.h"
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>

#include "kernels.h"
#include "plan.h"
#include "tile.h"

namespace qlb {

namespace {
thread_local std::string g_last_error;

// Multiprocessor count per device index, looked up on first use.
constexpr int kMaxDevices = 64;
std::atomic<int> g_sm_count[kMaxDevices];
}  // namespace

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
    int v = g_sm_count[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        g_sm_count[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

void fail(qlb_status code, const std::string& msg) { throw Error{code, msg}; }
void set_last_error(const std::string& msg) { g_last_error = msg; }

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(QLB_ERR_OOM, std::string(what) + ": out of device memory");
    }
    fail(QLB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void* DeviceBuffer::ensure(size_t bytes) {
    if (bytes <= cap && p) return p;
    release();
    size_t want = bytes < 256 ? 256 : bytes;
    check_cuda(cudaMalloc(&p, want), "cudaMalloc(scratch)");
    cap = want;
    return p;
}
void DeviceBuffer::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
void* PinnedBuffer::ensure(size_t bytes) {
    if (bytes <= cap && p) return p;
    release();
    size_t want = bytes < 4096 ? 4096 : bytes;
    check_cuda(cudaMallocHost(&p, want), "cudaMallocHost");
    cap = want;
    return p;
}
void PinnedBuffer::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

void state_allocate(qlb_state& sv, uint32_t n) {
    if (n > 34) fail(QLB_ERR_INVALID_ARG, "state vector: at most 34 qubits fit in one GPU's HBM");
    const uint64_t dim = uint64_t{1} << n;
    if (sv.d && sv.dim == dim) {
        sv.n = n;
        return;
    }
    state_free(sv);
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, dim * sizeof(float2)), "cudaMalloc(state)");
    sv.d = static_cast<float2*>(p);
    sv.n = n;
    sv.dim = dim;
}

void state_free(qlb_state& sv) {
    if (sv.d) cudaFree(sv.d);
    sv.d = nullptr;
    sv.n = 0;
    sv.dim = 0;
}

static constexpr uint64_t kStageElems = uint64_t{1} << 23;  // 8 Mi complex128 = 128 MiB

void state_upload_c128(qlb_state& sv, const double* amps, uint64_t dim, cudaStream_t s, DeviceBuffer& staging) {
    double2* st = static_cast<double2*>(staging.ensure(std::min(dim, kStageElems) * sizeof(double2)));
    for (uint64_t off = 0; off < dim; off += kStageElems) {
        const uint64_t cnt = std::min(kStageElems, dim - off);
        check_cuda(cudaMemcpyAsync(st, amps + 2 * off, cnt * sizeof(double2), cudaMemcpyHostToDevice, s), "H2D state");
        check_cuda(launch_c128_to_c64(st, sv.d + off, cnt, s), "c128->c64");
    }
    check_cuda(cudaStreamSynchronize(s), "upload sync");
}

void state_download_c128(const qlb_state& sv, double* out, cudaStream_t s, DeviceBuffer& staging) {
    double2* st = static_cast<double2*>(staging.ensure(std::min(sv.dim, kStageElems) * sizeof(double2)));
    for (uint64_t off = 0; off < sv.dim; off += kStageElems) {
        const uint64_t cnt = std::min(kStageElems, sv.dim - off);
        check_cuda(launch_c64_to_c128(sv.d + off, st, cnt, s), "c64->c128");
        check_cuda(cudaMemcpyAsync(out + 2 * off, st, cnt * sizeof(double2), cudaMemcpyDeviceToHost, s), "D2H state");
    }
    check_cuda(cudaStreamSynchronize(s), "download sync");
}

// ---------------------------------------------------------------------------
// Gate matrices (host, FP64 -> complex64)
// ---------------------------------------------------------------------------

Mat2f gate_matrix_1q(uint8_t type, float param) {
    const double r2 = 1.0 / std::sqrt(2.0);
    const double h = static_cast<double>(param) * 0.5, c = std::cos(h), s = std::sin(h);
    double m[8] = {1, 0, 0, 0, 0, 0, 1, 0};
    auto set = [&](double a, double b, double cc, double d, double e, double f, double g, double hh) {
        m[0] = a; m[1] = b; m[2] = cc; m[3] = d; m[4] = e; m[5] = f; m[6] = g; m[7] = hh;
    };
    switch (type) {
    case QLB_H: set(r2, 0, r2, 0, r2, 0, -r2, 0); break;
    case QLB_X: set(0, 0, 1, 0, 1, 0, 0, 0); break;
    case QLB_Y: set(0, 0, 0, -1, 0, 1, 0, 0); break;
    case QLB_Z: set(1, 0, 0, 0, 0, 0, -1, 0); break;
    case QLB_S: set(1, 0, 0, 0, 0, 0, 0, 1); break;
    case QLB_RX: set(c, 0, 0, -s, 0, -s, c, 0); break;
    case QLB_RY: set(c, 0, -s, 0, s, 0, c, 0); break;
    case QLB_RZ: set(std::cos(-h), std::sin(-h), 0, 0, 0, 0, std::cos(h), std::sin(h)); break;
    default: break;
    }
    Mat2f r;
    for (int i = 0; i < 4; ++i) r.m[i] = make_float2(static_cast<float>(m[2 * i]), static_cast<float>(m[2 * i + 1]));
    return r;
}

uint32_t instr_qubit(const qlb_gate_instr& in, uint32_t j) { return j < 4 ? in.qubits[j] : in.qubits_ext[j - 4]; }

// Validates one instruction against the state size and pool; returns its
// arity.  Throws QLB_ERR_UNKNOWN_GATE / QLB_ERR_INVALID_ARG.
uint32_t validate_instr(const qlb_gate_instr& in, uint32_t n, const qlb_pool_view* pool) {
    uint32_t k = 0;
    switch (in.type) {
    case QLB_H: case QLB_X: case QLB_Y: case QLB_Z: case QLB_S:
    case QLB_RX: case QLB_RY: case QLB_RZ: case QLB_MEASURE: k = 1; break;
    case QLB_CX: case QLB_SWAP: case QLB_CZ: case QLB_CP: case QLB_GLOBAL_SWAP: k = 2; break;
    case QLB_CCX: case QLB_CSWAP: k = 3; break;
    case QLB_UNITARY: case QLB_FUSED_BLOCK: {
        k = in.flags_arity & 0x0F;
        if (k < 1 || k > 6) fail(QLB_ERR_INVALID_ARG, "dense instruction arity must be 1..6");
        if (!pool || in.payload.matrix_idx >= pool->num_matrices)
            fail(QLB_ERR_INVALID_ARG, "matrix_idx out of range of the UnitaryPool");
        const qlb_matrix_entry& e = pool->metadata[in.payload.matrix_idx];
        if (e.num_elements != (1u << (2 * k)) || e.num_qubits != k ||
            uint64_t{e.offset} + e.num_elements > pool->num_elements)
            fail(QLB_ERR_INVALID_ARG, "UnitaryPool entry does not match the instruction arity");
        break;
    }
    case QLB_BARRIER: return 0;
    default: fail(QLB_ERR_UNKNOWN_GATE, "CUDAEngine: Unrecognized instruction type");
    }
    uint64_t seen = 0;
    for (uint32_t j = 0; j < k; ++j) {
        const uint32_t q = instr_qubit(in, j);
        if (q >= n) fail(QLB_ERR_INVALID_ARG, "qubit index out of range");
        if (seen & (uint64_t{1} << q)) fail(QLB_ERR_INVALID_ARG, "instruction repeats a qubit");
        seen |= uint64_t{1} << q;
    }
    return k;
}

// Reads (and clears) the flag the tile kernel raises when a bounded wait
// gives up; the stream must be idle.
void check_device_error(qlb_engine& e) {
    if (!e.err_flag.p) return;
    int flag = 0;
    check_cuda(cudaMemcpy(&flag, e.err_flag.p, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
    if (flag != 0) {
        check_cuda(cudaMemsetAsync(e.err_flag.p, 0, sizeof(int), e.stream), "clear error flag");
        fail(QLB_ERR_TIMEOUT, "a tile pass gave up waiting for its TMA copies; the state is undefined");
    }
}

double prob_one(qlb_engine& e, uint32_t mem_qubit) {
    const uint32_t cap = static_cast<uint32_t>(sm_count()) * 4u;
    double* part = static_cast<double*>(e.red_partial.ensure(cap * sizeof(double)));
    double* out = static_cast<double*>(e.red_out.ensure(64 * sizeof(double)));
    check_cuda(launch_prob_one(e.sv.d, e.sv.n, mem_qubit, part, cap, out, e.stream), "prob_one");
    double* h = static_cast<double*>(e.host_pinned.ensure(64 * sizeof(double)));
    check_cuda(cudaMemcpyAsync(h, out, sizeof(double), cudaMemcpyDeviceToHost, e.stream), "D2H prob");
    check_cuda(cudaStreamSynchronize(e.stream), "prob sync");
    return h[0];
}

// apply_measure (:617-671) with the reference's RNG draw and clamp.
void measure(qlb_engine& e, uint32_t mem_qubit) {
    const double p1 = prob_one(e, mem_qubit);
    const double r = e.dist(e.rng);
    const uint8_t outcome = (r < p1) ? 1 : 0;
    e.measurements.push_back(outcome);
    double p = outcome ? p1 : (1.0 - p1);
    if (p < 1e-12) p = 1e-12;
    const double inv = 1.0 / std::sqrt(p);
    check_cuda(launch_collapse(e.sv.d, e.sv.n, mem_qubit, outcome, static_cast<float>(inv), e.stream), "collapse");
}

// One plain instruction (already validated) whose qubits are memory qubits.
void apply_plain(qlb_engine& e, const qlb_gate_instr& in, const float2* mat) {
    float2* a = e.sv.d;
    const uint32_t n = e.sv.n;
    auto Q = [&](uint32_t j) { return instr_qubit(in, j); };
    auto bit = [](uint32_t q) { return uint64_t{1} << q; };
    cudaStream_t s = e.stream;
    switch (in.type) {
    case QLB_H: case QLB_Y: case QLB_RX: case QLB_RY:
        check_cuda(launch_apply_1q(a, n, Q(0), gate_matrix_1q(in.type, in.payload.param), s), "1q");
        break;
    case QLB_X: {
        uint32_t h[1] = {Q(0)};
        check_cuda(launch_swap_subspace(a, n, h, 1, 0, bit(Q(0)), s), "x");
        break;
    }
    case QLB_Z: case QLB_S: case QLB_RZ: {
        Mat2f m = gate_matrix_1q(in.type, in.payload.param);
        check_cuda(launch_apply_diag1(a, n, Q(0), m.m[0], m.m[3], s), "diag1");
        break;
    }
    case QLB_CX: {
        uint32_t h[2] = {Q(0), Q(1)};
        check_cuda(launch_swap_subspace(a, n, h, 2, bit(Q(0)), bit(Q(0)) | bit(Q(1)), s), "cx");
        break;
    }
    case QLB_SWAP: {
        uint32_t h[2] = {Q(0), Q(1)};
        check_cuda(launch_swap_subspace(a, n, h, 2, bit(Q(1)), bit(Q(0)), s), "swap");
        break;
    }
    case QLB_CZ: case QLB_CP: {
        uint32_t h[2] = {Q(0), Q(1)};
        float2 ph = make_float2(-1.f, 0.f);
        if (in.type == QLB_CP) {
            const double phi = static_cast<double>(in.payload.param);
            ph = make_float2(static_cast<float>(std::cos(phi)), static_cast<float>(std::sin(phi)));
        }
        check_cuda(launch_phase_mask(a, n, h, 2, bit(Q(0)) | bit(Q(1)), ph, s), "cphase");
        break;
    }
    case QLB_CCX: {
        uint32_t h[3] = {Q(0), Q(1), Q(2)};
        const uint64_t c = bit(Q(0)) | bit(Q(1));
        check_cuda(launch_swap_subspace(a, n, h, 3, c, c | bit(Q(2)), s), "ccx");
        break;
    }
    case QLB_CSWAP: {
        uint32_t h[3] = {Q(0), Q(1), Q(2)};
        const uint64_t c = bit(Q(0));
        check_cuda(launch_swap_subspace(a, n, h, 3, c | bit(Q(2)), c | bit(Q(1)), s), "cswap");
        break;
    }
    case QLB_UNITARY: case QLB_FUSED_BLOCK: {
        const uint32_t k = in.flags_arity & 0x0F;
        uint32_t q[6];
        for (uint32_t j = 0; j < k; ++j) q[j] = Q(j);
        check_cuda(launch_apply_dense(a, n, q, k, mat, s), "dense");
        break;
    }
    default: break;
    }
}

}  // namespace qlb

// ===========================================================================
// C ABI
// ===========================================================================

using namespace qlb;

namespace {

uint32_t log2_exact(uint64_t dim) {
    if (dim == 0 || (dim & (dim - 1)) != 0)
        fail(QLB_ERR_INVALID_ARG, "CUDAStateVector: Input state dimension must be a power of 2.");
    uint32_t n = 0;
    while ((uint64_t{1} << n) < dim) ++n;
    return n;
}

double device_norm_sq(const qlb_state& sv, cudaStream_t s, DeviceBuffer& part, DeviceBuffer& out, PinnedBuffer& host) {
    const uint32_t cap = static_cast<uint32_t>(sm_count()) * 4u;
    double* p = static_cast<double*>(part.ensure(cap * sizeof(double)));
    double* o = static_cast<double*>(out.ensure(64 * sizeof(double)));
    check_cuda(launch_norm_sq(sv.d, sv.dim, p, cap, o, s), "norm");
    double* h = static_cast<double*>(host.ensure(64 * sizeof(double)));
    check_cuda(cudaMemcpyAsync(h, o, sizeof(double), cudaMemcpyDeviceToHost, s), "D2H norm");
    check_cuda(cudaStreamSynchronize(s), "norm sync");
    return h[0];
}

// initialize(span) (cpu_state_vector.hpp:82-115): power-of-2 and norm
// checks (the norm in FP64 over the uploaded amplitudes); on failure the
// previous contents are kept.
void initialize_from(qlb_state& sv, const double* amps, uint64_t dim, cudaStream_t s, DeviceBuffer& staging,
                     DeviceBuffer& part, DeviceBuffer& out, PinnedBuffer& host) {
    need(amps, "amplitudes");
    const uint32_t n = log2_exact(dim);
    qlb_state fresh;
    state_allocate(fresh, n);
    try {
        state_upload_c128(fresh, amps, dim, s, staging);
        const double norm = device_norm_sq(fresh, s, part, out, host);
        if (std::fabs(norm - 1.0) > 1e-6)
            fail(QLB_ERR_NOT_NORMALIZED, "CUDAStateVector: Provided state vector is not normalized (norm squared != 1.0).");
    } catch (...) {
        state_free(fresh);
        throw;
    }
    state_free(sv);
    sv = fresh;
}

struct StandaloneScratch {
    DeviceBuffer staging, part, out;
    PinnedBuffer host;
};

cudaStream_t make_stream() {
    cudaStream_t s = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    return s;
}

}  // namespace

extern "C" {

const char* qlb_last_error(void) { return g_last_error.c_str(); }
const char* qlb_version(void) { return "qlassical_b200 0.1 (sm_100a)"; }

int qlb_set_device(int device) {
    return guarded([&] {
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
    });
}

int qlb_device_info(int* sm, uint64_t* free_b, uint64_t* total_b) {
    return guarded([&] {
        size_t f = 0, t = 0;
        check_cuda(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
        if (sm) *sm = sm_count();
        if (free_b) *free_b = f;
        if (total_b) *total_b = t;
    });
}

int qlb_selftest_bounded_wait(uint32_t limit_ms, int* gave_up) {
    return guarded([&] {
        need(gave_up, "gave_up");
        if (limit_ms == 0 || limit_ms > 2000) fail(QLB_ERR_INVALID_ARG, "limit_ms must be in 1..2000");
        DeviceBuffer flag;
        int* d = static_cast<int*>(flag.ensure(256));
        check_cuda(cudaMemset(d, 0, sizeof(int)), "flag clear");
        check_cuda(launch_wait_selftest(uint64_t{limit_ms} * 1000000ull, d, nullptr), "wait self-test");
        check_cuda(cudaStreamSynchronize(nullptr), "wait self-test sync");
        int h = 0;
        check_cuda(cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost), "flag D2H");
        *gave_up = h;
    });
}

// ---- state ---------------------------------------------------------------

int qlb_state_create(qlb_state_t* out) {
    return guarded([&] {
        need(out, "out");
        *out = new qlb_state();
    });
}
int qlb_state_destroy(qlb_state_t sv) {
    return guarded([&] {
        if (!sv) return;
        state_free(*sv);
        delete sv;
    });
}
int qlb_state_initialize(qlb_state_t sv, uint32_t n) {
    return guarded([&] {
        need(sv, "state");
        state_allocate(*sv, n);
        check_cuda(launch_init_zero(sv->d, sv->dim, nullptr), "init");
        check_cuda(cudaStreamSynchronize(nullptr), "init sync");
    });
}
int qlb_state_initialize_from(qlb_state_t sv, const double* amps, uint64_t dim) {
    return guarded([&] {
        need(sv, "state");
        StandaloneScratch sc;
        initialize_from(*sv, amps, dim, nullptr, sc.staging, sc.part, sc.out, sc.host);
    });
}
int qlb_state_num_qubits(qlb_state_t sv, uint32_t* out) {
    return guarded([&] { need(sv, "state"); need(out, "out"); *out = sv->n; });
}
int qlb_state_dimension(qlb_state_t sv, uint64_t* out) {
    return guarded([&] { need(sv, "state"); need(out, "out"); *out = sv->dim; });
}
int qlb_state_empty(qlb_state_t sv, int* out) {
    return guarded([&] { need(sv, "state"); need(out, "out"); *out = sv->dim == 0; });
}
int qlb_state_download(qlb_state_t sv, double* out, uint64_t dim) {
    return guarded([&] {
        need(sv, "state");
        need(out, "out");
        if (sv->dim == 0) fail(QLB_ERR_STATE, "state vector is empty");
        if (dim != sv->dim) fail(QLB_ERR_INVALID_ARG, "output size does not match the state dimension");
        StandaloneScratch sc;
        state_download_c128(*sv, out, nullptr, sc.staging);
    });
}
int qlb_state_device_ptr(qlb_state_t sv, void** out) {
    return guarded([&] { need(sv, "state"); need(out, "out"); *out = sv->d; });
}

// ---- engine --------------------------------------------------------------

static qlb_engine* new_engine(int has_seed, uint64_t seed, uint64_t reserve) {
    auto* e = new qlb_engine();
    try {
        e->stream = make_stream();
    } catch (...) {
        delete e;
        throw;
    }
    if (has_seed) {
        e->rng.seed(seed);
    } else {
        std::random_device rd;
        e->rng.seed(rd());
    }
    if (reserve) e->measurements.reserve(reserve);
    return e;
}

static void delete_engine(qlb_engine* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    state_free(e->sv);
    e->red_partial.release();
    e->red_out.release();
    e->err_flag.release();
    e->staging.release();
    e->host_pinned.release();
    e->host_prog.release();
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int qlb_engine_create(qlb_engine_t* out, uint32_t n, int has_seed, uint64_t seed, uint64_t reserve) {
    return guarded([&] {
        need(out, "out");
        qlb_engine* e = new_engine(has_seed, seed, reserve);
        try {
            state_allocate(e->sv, n);
            check_cuda(launch_init_zero(e->sv.d, e->sv.dim, e->stream), "init");
            check_cuda(cudaStreamSynchronize(e->stream), "init sync");
        } catch (...) {
            delete_engine(e);
            throw;
        }
        *out = e;
    });
}

int qlb_engine_create_from_amplitudes(qlb_engine_t* out, const double* amps, uint64_t dim, int has_seed,
                                      uint64_t seed, uint64_t reserve) {
    return guarded([&] {
        need(out, "out");
        qlb_engine* e = new_engine(has_seed, seed, reserve);
        try {
            initialize_from(e->sv, amps, dim, e->stream, e->staging, e->red_partial, e->red_out, e->host_pinned);
        } catch (...) {
            delete_engine(e);
            throw;
        }
        *out = e;
    });
}

// CPUOpenMPEngine(CPUStateVector&&) (:105-107): takes the device buffer,
// leaves `sv` empty; the RNG keeps its default seed, as in the reference.
int qlb_engine_create_from_state(qlb_engine_t* out, qlb_state_t sv) {
    return guarded([&] {
        need(out, "out");
        need(sv, "state");
        auto* e = new qlb_engine();
        try {
            e->stream = make_stream();
        } catch (...) {
            delete e;
            throw;
        }
        e->sv = *sv;
        *sv = qlb_state{};
        *out = e;
    });
}

int qlb_engine_destroy(qlb_engine_t e) {
    return guarded([&] { delete_engine(e); });
}

int qlb_engine_set_state_vector(qlb_engine_t e, qlb_state_t sv) {
    return guarded([&] {
        need(e, "engine");
        need(sv, "state");
        check_cuda(cudaStreamSynchronize(e->stream), "sync");
        state_free(e->sv);
        e->sv = *sv;
        *sv = qlb_state{};
    });
}

int qlb_engine_extract_state_vector(qlb_engine_t e, qlb_state_t out) {
    return guarded([&] {
        need(e, "engine");
        need(out, "state");
        check_cuda(cudaStreamSynchronize(e->stream), "sync");
        state_free(*out);
        *out = e->sv;
        e->sv = qlb_state{};
    });
}

int qlb_engine_reset(qlb_engine_t e) {
    return guarded([&] {
        need(e, "engine");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        check_cuda(launch_init_zero(e->sv.d, e->sv.dim, e->stream), "init");
        e->measurements.clear();
    });
}

int qlb_engine_reset_to(qlb_engine_t e, const double* amps, uint64_t dim) {
    return guarded([&] {
        need(e, "engine");
        initialize_from(e->sv, amps, dim, e->stream, e->staging, e->red_partial, e->red_out, e->host_pinned);
        e->measurements.clear();
    });
}

int qlb_engine_set_seed(qlb_engine_t e, uint64_t seed) {
    return guarded([&] { need(e, "engine"); e->rng.seed(seed); });
}
int qlb_engine_reserve_measurements(qlb_engine_t e, uint64_t count) {
    return guarded([&] { need(e, "engine"); e->measurements.reserve(count); });
}
int qlb_engine_measurements(qlb_engine_t e, const uint8_t** data, uint64_t* count) {
    return guarded([&] {
        need(e, "engine");
        need(data, "data");
        need(count, "count");
        *data = e->measurements.data();
        *count = e->measurements.size();
    });
}

int qlb_engine_execute(qlb_engine_t e, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool) {
    return guarded([&] {
        need(e, "engine");
        if (count && !prog) fail(QLB_ERR_INVALID_ARG, "program is null");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        for (uint64_t i = 0; i < count; ++i) validate_instr(prog[i], e->sv.n, pool);
        // the plan's device image goes to a buffer the engine keeps, so a
        // call allocates and frees no device memory once it has grown
        std::unique_ptr<qlb_plan> p(compile_plan(*e, prog, count, pool, &e->exec_plan));
        e->stats = p->stats;
        run_plan(*e, *p);
        // the kernels that read the plan image must finish before the next
        // call reuses the buffer
        check_cuda(cudaStreamSynchronize(e->stream), "execute sync");
        check_device_error(*e);
    });
}

int qlb_engine_compile(qlb_engine_t e, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool,
                       qlb_plan_t* out) {
    return guarded([&] {
        need(e, "engine");
        need(out, "out");
        if (count && !prog) fail(QLB_ERR_INVALID_ARG, "program is null");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        for (uint64_t i = 0; i < count; ++i) validate_instr(prog[i], e->sv.n, pool);
        *out = compile_plan(*e, prog, count, pool);
        check_cuda(cudaStreamSynchronize(e->stream), "compile sync");
    });
}

int qlb_engine_run(qlb_engine_t e, qlb_plan_t plan) {
    return guarded([&] {
        need(e, "engine");
        need(plan, "plan");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        e->stats = plan->stats;
        run_plan(*e, *plan);
    });
}

int qlb_describe_plan(uint32_t n, int mode, int physical, const qlb_gate_instr* prog, uint64_t count,
                      const qlb_pool_view* pool, char* out, uint64_t cap, uint64_t* needed) {
    return qlb_describe_plan_opts(n, mode, physical, kTileLow, 1, prog, count, pool, out, cap, needed);
}

int qlb_describe_plan_opts(uint32_t n, int mode, int physical, int tile_low, int tc_chain, const qlb_gate_instr* prog,
                           uint64_t count, const qlb_pool_view* pool, char* out, uint64_t cap, uint64_t* needed) {
    return guarded([&] {
        if (count && !prog) fail(QLB_ERR_INVALID_ARG, "program is null");
        if (n > 34) fail(QLB_ERR_INVALID_ARG, "at most 34 qubits");
        if (mode < QLB_MODE_PLAIN || mode > QLB_MODE_TILED_TC) fail(QLB_ERR_INVALID_ARG, "unknown execution mode");
        for (uint64_t i = 0; i < count; ++i) validate_instr(prog[i], n, pool);
        const std::string js =
            describe_plan_json(PlanConfig{n, mode, physical, 10.0, tc_chain != 0, tile_low}, prog, count, pool);
        if (needed) *needed = js.size() + 1;
        if (out && cap) {
            const size_t m = std::min<size_t>(cap - 1, js.size());
            std::memcpy(out, js.data(), m);
            out[m] = '\0';
        }
    });
}

int qlb_plan_stats(qlb_plan_t plan, qlb_exec_stats* out) {
    return guarded([&] { need(plan, "plan"); need(out, "out"); *out = plan->stats; });
}

int qlb_plan_destroy(qlb_plan_t plan) {
    return guarded([&] { delete plan; });
}

int qlb_engine_state(qlb_engine_t e, double* out, uint64_t dim) {
    return guarded([&] {
        need(e, "engine");
        need(out, "out");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        if (dim != e->sv.dim) fail(QLB_ERR_INVALID_ARG, "output size does not match the state dimension");
        state_download_c128(e->sv, out, e->stream, e->staging);
    });
}

int qlb_engine_num_qubits(qlb_engine_t e, uint32_t* out) {
    return guarded([&] { need(e, "engine"); need(out, "out"); *out = e->sv.n; });
}
int qlb_engine_set_mode(qlb_engine_t e, int mode) {
    return guarded([&] {
        need(e, "engine");
        if (mode < QLB_MODE_PLAIN || mode > QLB_MODE_TILED_TC) fail(QLB_ERR_INVALID_ARG, "unknown execution mode");
        e->mode = mode;
    });
}
int qlb_engine_set_option(qlb_engine_t e, int key, int64_t value) {
    return guarded([&] {
        need(e, "engine");
        if (key == QLB_OPT_PHYSICAL_GLOBAL_SWAP) {
            e->physical_global_swap = value != 0;
        } else if (key == QLB_OPT_TC_MIN_COST) {
            if (value < 0) fail(QLB_ERR_INVALID_ARG, "QLB_OPT_TC_MIN_COST must be >= 0");
            e->tc_min_cost = static_cast<double>(value) / 100.0;
        } else if (key == QLB_OPT_TC_CHAIN) {
            e->tc_chain = value != 0;
        } else if (key == QLB_OPT_TILE_LOW) {
            if (value < kTileLow || value > kTileLowMax)
                fail(QLB_ERR_INVALID_ARG, "QLB_OPT_TILE_LOW must be in 3..6");
            e->tile_low = static_cast<int>(value);
        } else {
            fail(QLB_ERR_INVALID_ARG, "unknown engine option");
        }
    });
}
int qlb_engine_get_mode(qlb_engine_t e, int* mode) {
    return guarded([&] { need(e, "engine"); need(mode, "mode"); *mode = e->mode; });
}
int qlb_engine_synchronize(qlb_engine_t e) {
    return guarded([&] {
        need(e, "engine");
        check_cuda(cudaStreamSynchronize(e->stream), "sync");
        check_device_error(*e);
    });
}
int qlb_engine_device_state(qlb_engine_t e, void** out) {
    return guarded([&] { need(e, "engine"); need(out, "out"); *out = e->sv.d; });
}
int qlb_engine_stream(qlb_engine_t e, void** out) {
    return guarded([&] { need(e, "engine"); need(out, "out"); *out = e->stream; });
}
int qlb_engine_last_stats(qlb_engine_t e, qlb_exec_stats* out) {
    return guarded([&] { need(e, "engine"); need(out, "out"); *out = e->stats; });
}

int qlb_engine_norm_sq(qlb_engine_t e, double* out) {
    return guarded([&] {
        need(e, "engine");
        need(out, "out");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        *out = device_norm_sq(e->sv, e->stream, e->red_partial, e->red_out, e->host_pinned);
    });
}

int qlb_engine_prob_one(qlb_engine_t e, uint32_t qubit, double* out) {
    return guarded([&] {
        need(e, "engine");
        need(out, "out");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        if (qubit >= e->sv.n) fail(QLB_ERR_INVALID_ARG, "qubit index out of range");
        *out = prob_one(*e, qubit);
    });
}

int qlb_engine_expect_z(qlb_engine_t e, double* out, uint32_t nq) {
    return guarded([&] {
        need(e, "engine");
        need(out, "out");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        if (nq != e->sv.n) fail(QLB_ERR_INVALID_ARG, "output length must equal the number of qubits");
        const uint32_t n = e->sv.n;
        const uint32_t cap = marginals_partial_size(n);
        double* part = static_cast<double*>(e->red_partial.ensure(static_cast<size_t>(cap) * sizeof(double)));
        double* o = static_cast<double*>(e->red_out.ensure(64 * sizeof(double)));
        check_cuda(launch_qubit_marginals(e->sv.d, n, part, cap, o, e->stream), "marginals");
        double* h = static_cast<double*>(e->host_pinned.ensure(64 * sizeof(double)));
        check_cuda(cudaMemcpyAsync(h, o, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, e->stream), "D2H");
        check_cuda(cudaStreamSynchronize(e->stream), "expect sync");
        const double tot = h[0];
        for (uint32_t q = 0; q < n; ++q) out[q] = tot - 2.0 * h[1 + q];
    });
}

int qlb_engine_amplitudes_at(qlb_engine_t e, const uint64_t* indices, uint64_t count, double* out_c128) {
    return guarded([&] {
        need(e, "engine");
        if (count && (!indices || !out_c128)) fail(QLB_ERR_INVALID_ARG, "indices / out is null");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        for (uint64_t i = 0; i < count; ++i)
            if (indices[i] >= e->sv.dim) fail(QLB_ERR_INVALID_ARG, "amplitude index out of range");
        if (count == 0) return;
        char* buf = static_cast<char*>(e->staging.ensure(count * (sizeof(uint64_t) + 2 * sizeof(double)) + 256));
        auto* d_idx = reinterpret_cast<uint64_t*>(buf);
        auto* d_out = reinterpret_cast<double2*>(buf + ((count * sizeof(uint64_t) + 255) & ~size_t{255}));
        check_cuda(cudaMemcpyAsync(d_idx, indices, count * sizeof(uint64_t), cudaMemcpyHostToDevice, e->stream), "H2D");
        check_cuda(launch_gather(e->sv.d, d_idx, count, d_out, e->stream), "gather");
        check_cuda(cudaMemcpyAsync(out_c128, d_out, count * 2 * sizeof(double), cudaMemcpyDeviceToHost, e->stream),
                   "D2H");
        check_cuda(cudaStreamSynchronize(e->stream), "gather sync");
    });
}

int qlb_engine_sample(qlb_engine_t e, uint64_t seed, uint64_t shots, uint64_t* out) {
    return guarded([&] {
        need(e, "engine");
        if (shots && !out) fail(QLB_ERR_INVALID_ARG, "out is null");
        if (e->sv.dim == 0) fail(QLB_ERR_STATE, "engine has no state vector");
        const uint64_t scratch = sample_scratch_doubles(e->sv.n);
        double* cs = static_cast<double*>(e->red_partial.ensure(scratch * sizeof(double)));
        uint64_t* d_out = static_cast<uint64_t*>(e->staging.ensure((shots ? shots : 1) * sizeof(uint64_t)));
        check_cuda(launch_sample(e->sv.d, e->sv.n, seed, shots, cs, d_out, e->stream), "sample");
        if (shots)
            check_cuda(cudaMemcpyAsync(out, d_out, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, e->stream), "D2H");
        check_cuda(cudaStreamSynchronize(e->stream), "sample sync");
    });
}

}  // extern "C"

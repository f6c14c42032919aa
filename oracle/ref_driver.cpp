// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C ABI over the unmodified Qlassical reference (compiled from its own
// headers, see oracle/Makefile) so that tests/ and the CPU-baseline leg of
// bench.py can run the reference engine and middle end through ctypes:
//   qlref_execute       -> CPUOpenMPEngine(init)::execute (cpu_openmp_engine.hpp:65-107, 143-225)
//   qlref_transpile     -> Middleware::transpile(module, CPU_OPENMP, cfg) (middleware.hpp:466-524)
//   qlref_time_execute  -> the reference benchmark loop (bench_hw_awareness.cpp:100-107)
#include <chrono>
#include <complex>
#include <cstring>
#include <memory>
#include <optional>
#include <span>
#include <vector>

#include <omp.h>

#include <backend/cpu_openmp_engine.hpp>
#include <frontend/frontend.hpp>
#include <middleware/middleware.hpp>

using namespace qlassical;

// The ctypes side passes the reference's own GateInstr records and a plain
// view of a UnitaryPool (complex128 data + MatrixEntry records).
using qlb_gate_instr = GateInstr;
using qlb_matrix_entry = UnitaryPool::MatrixEntry;
struct qlb_pool_view {
    const double* data;
    uint64_t num_elements;
    const qlb_matrix_entry* metadata;
    uint64_t num_matrices;
};
static_assert(sizeof(GateInstr) == 16, "GateInstr layout");
static_assert(sizeof(UnitaryPool::MatrixEntry) == 12, "MatrixEntry layout");

namespace {

UnitaryPool make_pool(const qlb_pool_view* pv) {
    UnitaryPool pool;
    if (!pv || pv->num_matrices == 0) return pool;
    auto* c = reinterpret_cast<const std::complex<double>*>(pv->data);
    pool.data.assign(c, c + pv->num_elements);
    pool.metadata.resize(pv->num_matrices);
    std::memcpy(pool.metadata.data(), pv->metadata, pv->num_matrices * sizeof(qlb_matrix_entry));
    return pool;
}

std::span<const GateInstr> as_program(const qlb_gate_instr* p, uint64_t n) {
    return {reinterpret_cast<const GateInstr*>(p), static_cast<std::size_t>(n)};
}

struct RefModule {
    IRModule module;
};

}  // namespace

extern "C" {

int qlref_num_threads(void) { return omp_get_max_threads(); }

// Runs `prog` on a fresh engine (|0..0> if init == nullptr, else the given
// complex128 amplitudes) and copies the final state out.
int qlref_execute(uint32_t n, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pv,
                  const double* init, int has_seed, uint64_t seed, double* out_state,
                  uint8_t* meas, uint64_t meas_cap, uint64_t* meas_count) {
    try {
        std::optional<uint64_t> s = has_seed ? std::optional<uint64_t>(seed) : std::nullopt;
        std::unique_ptr<backend::CPUOpenMPEngine> eng;
        if (init) {
            auto* c = reinterpret_cast<const std::complex<double>*>(init);
            eng = std::make_unique<backend::CPUOpenMPEngine>(
                std::span<const std::complex<double>>(c, std::size_t{1} << n), s, 0);
        } else {
            eng = std::make_unique<backend::CPUOpenMPEngine>(n, s, 0);
        }
        UnitaryPool pool = make_pool(pv);
        eng->execute(as_program(prog, count), pool);
        auto st = eng->state();
        std::memcpy(out_state, st.data(), st.size() * sizeof(std::complex<double>));
        const auto& m = eng->measurements();
        if (meas_count) *meas_count = m.size();
        for (std::size_t i = 0; i < m.size() && i < meas_cap; ++i) meas[i] = m[i];
        return 0;
    } catch (const std::invalid_argument&) {
        return 1;
    } catch (const std::runtime_error&) {
        return 4;
    } catch (...) {
        return 3;
    }
}

// Reference transpilation; returns an owning handle (nullptr on error).
void* qlref_transpile(uint32_t n, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pv,
                      int fusion, int hw, int cost_model, uint32_t numa_penalty, uint32_t swap_penalty,
                      int k_safe) {
    try {
        auto* h = new RefModule{IRModule(n)};
        auto in = as_program(prog, count);
        h->module.gate_stream.assign(in.begin(), in.end());
        h->module.unitary_pool = make_pool(pv);
        TranspilerConfig cfg;
        cfg.enable_gate_fusion = fusion != 0;
        cfg.enable_hw_awareness = hw != 0;
        cfg.cost_model_type = cost_model == 1 ? CostModelType::GREEDY : CostModelType::THRESHOLD;
        cfg.numa_penalty = numa_penalty;
        cfg.swap_penalty = swap_penalty;
        if (k_safe >= 0) cfg.k_safe = static_cast<uint16_t>(k_safe);
        Middleware mw;
        mw.transpile(h->module, Backend::CPU_OPENMP, cfg);
        return h;
    } catch (...) {
        return nullptr;
    }
}

uint64_t qlref_module_count(void* h) { return static_cast<RefModule*>(h)->module.gate_stream.size(); }
uint64_t qlref_module_pool_elements(void* h) { return static_cast<RefModule*>(h)->module.unitary_pool.data.size(); }
uint64_t qlref_module_pool_matrices(void* h) { return static_cast<RefModule*>(h)->module.unitary_pool.metadata.size(); }
void qlref_module_copy(void* h, qlb_gate_instr* prog, double* pool_data, qlb_matrix_entry* meta) {
    auto& m = static_cast<RefModule*>(h)->module;
    std::memcpy(prog, m.gate_stream.data(), m.gate_stream.size() * sizeof(GateInstr));
    std::memcpy(pool_data, m.unitary_pool.data.data(), m.unitary_pool.data.size() * sizeof(std::complex<double>));
    std::memcpy(meta, m.unitary_pool.metadata.data(), m.unitary_pool.metadata.size() * sizeof(qlb_matrix_entry));
}
void qlref_module_free(void* h) { delete static_cast<RefModule*>(h); }

// Wall-clock seconds of `reps` timed execute() calls, each after an untimed
// reset(), exactly like the reference benchmark loop.  Returns the mean.
double qlref_time_execute(uint32_t n, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pv,
                          int reps) {
    try {
        backend::CPUOpenMPEngine eng(n, std::optional<uint64_t>(1), 0);
        UnitaryPool pool = make_pool(pv);
        double total = 0.0;
        for (int r = 0; r < reps; ++r) {
            eng.reset();
            auto t0 = std::chrono::steady_clock::now();
            eng.execute(as_program(prog, count), pool);
            auto t1 = std::chrono::steady_clock::now();
            total += std::chrono::duration<double>(t1 - t0).count();
        }
        return total / (reps > 0 ? reps : 1);
    } catch (...) {
        return -1.0;
    }
}

}  // extern "C"

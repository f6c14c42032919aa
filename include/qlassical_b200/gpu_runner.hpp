// gpu_runner.hpp -- the GPU middle end and orchestrator for the C++ drop-in.
//
//   GPUTopology        HardwareTopology (hw_topology.hpp:27-54) whose safe
//                      qubit limit is the tile window of the B200 kernels
//   transpile_gpu      Middleware::transpile_gpu (middleware.hpp:866, empty in
//                      the reference) over qlb_transpile_gpu; honours the
//                      reference's TranspilerConfig, including custom cost models
//   GPUCircuitRunner   CircuitRunner (circuit_runner.hpp:50-261) for
//                      Backend::GPU: blocks hand the state over on the device
#pragma once

#include <cmath>
#include <cstring>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <frontend/frontend.hpp>
#include <middleware/middleware.hpp>

#include "cuda_engine.hpp"

namespace qlassical::middleware {

// The base class computes floor(log2(0.85 * bytes / 16)); the GPU's locality
// domain is one on-chip tile of 2^13 amplitudes, so it reports the byte
// count for which that formula yields the tile width.
class GPUTopology : public HardwareTopology {
public:
    GPUTopology() {
        uint32_t k = 13;
        qlb_gpu_safe_qubit_limit(&k);
        tile_qubits_ = k;
    }
    std::size_t get_numa_memory_size_bytes() const override {
        return static_cast<std::size_t>(std::ceil(16.0 * std::ldexp(1.0, static_cast<int>(tile_qubits_)) / 0.85));
    }
    uint32_t get_numa_nodes_count() const override { return 1; }
    uint32_t tile_qubits() const noexcept { return tile_qubits_; }

private:
    uint32_t tile_qubits_ = 13;
};

namespace b200_detail {
inline int cost_model_trampoline(void* ctx, const uint32_t* freq, const uint16_t* l2p, const uint16_t* p2l,
                                 uint32_t n, uint16_t* active, uint16_t* victim) {
    const auto* model = static_cast<const WindowingCostModel*>(ctx);
    auto r = model->evaluate_swap(std::span<const uint32_t>(freq, n), std::span<const uint16_t>(l2p, n),
                                  std::span<const uint16_t>(p2l, n));
    if (!r) return 0;
    *active = r->first;
    *victim = r->second;
    return 1;
}
}  // namespace b200_detail

// Transpiles `module` in place for the B200 engine.  max_fusion_qubits is
// the GPU's fusion width (5 fits the register tile; the reference uses 4).
inline void transpile_gpu(IRModule& module, const TranspilerConfig& config = {}, int max_fusion_qubits = 5) {
    qlb_transpile_config c;
    qlb_transpile_config_default(&c);
    c.enable_gate_fusion = config.enable_gate_fusion;
    c.enable_hw_awareness = config.enable_hw_awareness;
    c.cost_model_type = static_cast<int>(config.cost_model_type);
    c.numa_penalty = config.numa_penalty;
    c.swap_penalty = config.swap_penalty;
    c.max_fusion_qubits = max_fusion_qubits;
    if (config.custom_cost_model) {
        c.custom_cost_model = &b200_detail::cost_model_trampoline;
        c.custom_cost_model_ctx = config.custom_cost_model.get();
        c.k_safe = config.k_safe.value_or(config.custom_cost_model->get_k_safe());
    } else {
        if (config.cost_model_type == CostModelType::CUSTOM)
            throw std::invalid_argument("TranspilerConfig: CostModelType::CUSTOM specified but custom_cost_model is null.");
        c.k_safe = config.k_safe.has_value() ? static_cast<int>(*config.k_safe)
                                             : static_cast<int>(GPUTopology().get_safe_qubit_limit());
    }
    const qlb_pool_view pv = backend::b200_detail::pool_view(module.unitaries());
    qlb_module_t out = nullptr;
    backend::b200_detail::check(qlb_transpile_gpu(reinterpret_cast<const qlb_gate_instr*>(module.gate_stream.data()),
                                                  module.gate_stream.size(), &pv, module.num_qubits, &c, &out));
    const qlb_gate_instr* prog = nullptr;
    uint64_t count = 0;
    qlb_pool_view pool{};
    qlb_module_program(out, &prog, &count);
    qlb_module_pool(out, &pool);
    IRModule result(module.num_qubits);
    result.gate_stream.resize(count);
    if (count) std::memcpy(static_cast<void*>(result.gate_stream.data()), prog, count * sizeof(GateInstr));
    const auto* data = reinterpret_cast<const std::complex<double>*>(pool.data);
    result.unitary_pool.data.assign(data, data + pool.num_elements);
    result.unitary_pool.metadata.resize(pool.num_matrices);
    if (pool.num_matrices)
        std::memcpy(static_cast<void*>(result.unitary_pool.metadata.data()), pool.metadata, pool.num_matrices * sizeof(qlb_matrix_entry));
    qlb_module_destroy(out);
    module = std::move(result);
}

}  // namespace qlassical::middleware

namespace qlassical {

// CircuitRunner for Backend::GPU.  Same block pipeline as
// CircuitRunner::run (circuit_runner.hpp:112-193): release -> transpile ->
// first block allocates, later blocks move the device state vector -> execute.
class GPUCircuitRunner {
public:
    explicit GPUCircuitRunner(std::shared_ptr<QuantumCircuit> circuit, middleware::TranspilerConfig config = {})
        : config_(std::move(config)) {
        if (!circuit) throw std::invalid_argument("CircuitRunner: circuit shared pointer cannot be null");
        circuits_.push_back(std::move(circuit));
    }
    explicit GPUCircuitRunner(std::vector<std::shared_ptr<QuantumCircuit>> circuits,
                              middleware::TranspilerConfig config = {})
        : circuits_(std::move(circuits)), config_(std::move(config)) {
        if (circuits_.empty()) throw std::invalid_argument("CircuitRunner: circuit block sequence cannot be empty");
        for (std::size_t i = 0; i < circuits_.size(); ++i)
            if (!circuits_[i])
                throw std::invalid_argument("CircuitRunner: null circuit pointer found at block index " +
                                            std::to_string(i));
    }

    void run() {
        backend::CUDAStateVector previous;
        bool first = true;
        for (std::size_t b = 0; b < circuits_.size(); ++b) {
            IRModule module = std::move(*circuits_[b]).release();
            middleware::transpile_gpu(module, config_);
            const uint32_t nq = module.num_qubits;
            std::unique_ptr<backend::CUDAEngine> engine;
            if (first) {
                engine = std::make_unique<backend::CUDAEngine>(nq);
                first = false;
            } else {
                if (previous.num_qubits() != nq)
                    throw std::invalid_argument("CircuitRunner::run: qubit count mismatch between block " +
                                                std::to_string(b - 1) + " (" + std::to_string(previous.num_qubits()) +
                                                " qubits) and block " + std::to_string(b) + " (" +
                                                std::to_string(nq) + " qubits)");
                engine = std::make_unique<backend::CUDAEngine>(std::move(previous));
            }
            engine->execute(module);
            if (b + 1 == circuits_.size()) engine_ = std::move(engine);
            else previous = std::move(*engine).extract_state_vector();
        }
    }

    [[nodiscard]] std::span<const std::complex<double>> state() const {
        if (!engine_) throw std::runtime_error("CircuitRunner::state: cannot inspect state before calling run()");
        return engine_->state();
    }
    [[nodiscard]] uint32_t num_qubits() const {
        if (!engine_)
            throw std::runtime_error("CircuitRunner::num_qubits: cannot inspect qubit count before calling run()");
        return engine_->num_qubits();
    }
    [[nodiscard]] const backend::CUDAEngine* engine() const noexcept { return engine_.get(); }
    [[nodiscard]] std::size_t num_blocks() const noexcept { return circuits_.size(); }
    [[nodiscard]] const std::vector<std::shared_ptr<QuantumCircuit>>& circuits() const noexcept { return circuits_; }
    [[nodiscard]] const middleware::TranspilerConfig& transpiler_config() const noexcept { return config_; }
    [[nodiscard]] Backend backend() const noexcept { return Backend::GPU; }

private:
    std::vector<std::shared_ptr<QuantumCircuit>> circuits_;
    middleware::TranspilerConfig config_;
    std::unique_ptr<backend::CUDAEngine> engine_;
};

}  // namespace qlassical

// cuda_engine.hpp -- C++20 drop-in for Qlassical: CUDAStateVector and
// CUDAEngine implement the reference's own StateVector
// (include/backend/state_vector.hpp:17-47) and ExecutionEngine
// (include/backend/execution_engine.hpp:20-79) interfaces on top of the C ABI
// in qlassical_b200.h, with the members CPUStateVector / CPUOpenMPEngine
// expose (cpu_state_vector.hpp:24-162, cpu_openmp_engine.hpp:51-247) and
// the reference's exception types:
//   QLB_ERR_INVALID_ARG / QLB_ERR_NOT_NORMALIZED -> std::invalid_argument
//   QLB_ERR_OOM                                  -> std::bad_alloc
//   QLB_ERR_UNKNOWN_GATE, QLB_ERR_CUDA, others   -> std::runtime_error
//
// Compile inside the reference's include tree (-I <qlassical>/include, plus
// its Eigen and OpenMP flags) and link libqlassical_b200.so.
// ExecutionEngine::execute(const IRModule&) is declared by the reference but
// defined only in cpu_openmp_engine.hpp (:678-680), so that header is
// included here too: every translation unit sees the one definition.
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <new>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <backend/cpu_openmp_engine.hpp>
#include <backend/execution_engine.hpp>
#include <backend/state_vector.hpp>
#include <frontend/frontend.hpp>

#include "../qlassical_b200.h"

namespace qlassical::backend {

namespace b200_detail {

inline void check(int status) {
    if (status == QLB_OK) return;
    const std::string msg = qlb_last_error();
    switch (status) {
    case QLB_ERR_INVALID_ARG:
    case QLB_ERR_NOT_NORMALIZED: throw std::invalid_argument(msg);
    case QLB_ERR_OOM: throw std::bad_alloc();
    default: throw std::runtime_error(msg);
    }
}

static_assert(sizeof(GateInstr) == sizeof(qlb_gate_instr), "GateInstr and qlb_gate_instr must match");
static_assert(sizeof(UnitaryPool::MatrixEntry) == sizeof(qlb_matrix_entry), "MatrixEntry layout");

inline qlb_pool_view pool_view(const UnitaryPool& pool) {
    return qlb_pool_view{reinterpret_cast<const double*>(pool.data.data()), pool.data.size(),
                         reinterpret_cast<const qlb_matrix_entry*>(pool.metadata.data()), pool.metadata.size()};
}

}  // namespace b200_detail

// complex64 state vector resident in HBM (move-only, like CPUStateVector).
class CUDAStateVector final : public StateVector {
public:
    using Amplitude = std::complex<double>;

    CUDAStateVector() { b200_detail::check(qlb_state_create(&h_)); }
    ~CUDAStateVector() override {
        if (h_) qlb_state_destroy(h_);
    }
    CUDAStateVector(CUDAStateVector&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    CUDAStateVector& operator=(CUDAStateVector&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    CUDAStateVector(const CUDAStateVector&) = delete;
    CUDAStateVector& operator=(const CUDAStateVector&) = delete;

    void initialize(uint32_t num_qubits) override { b200_detail::check(qlb_state_initialize(h_, num_qubits)); }
    void initialize(std::span<const Amplitude> amps) override {
        b200_detail::check(qlb_state_initialize_from(h_, reinterpret_cast<const double*>(amps.data()), amps.size()));
    }
    [[nodiscard]] uint32_t num_qubits() const noexcept override {
        uint32_t n = 0;
        if (h_) qlb_state_num_qubits(h_, &n);
        return n;
    }
    [[nodiscard]] std::size_t dimension() const noexcept override {
        uint64_t d = 0;
        if (h_) qlb_state_dimension(h_, &d);
        return static_cast<std::size_t>(d);
    }
    [[nodiscard]] bool empty() const noexcept override { return dimension() == 0; }

    // Device -> host copy, widened to complex128.
    [[nodiscard]] std::vector<Amplitude> amplitudes() const {
        std::vector<Amplitude> out(dimension());
        if (!out.empty()) b200_detail::check(qlb_state_download(h_, reinterpret_cast<double*>(out.data()), out.size()));
        return out;
    }
    [[nodiscard]] qlb_state_t handle() const noexcept { return h_; }

private:
    qlb_state_t h_ = nullptr;
};

// ExecutionEngine on one B200 GPU.
class CUDAEngine final : public ExecutionEngine {
public:
    using ExecutionEngine::execute;
    enum class Mode : int { Plain = QLB_MODE_PLAIN, Tiled = QLB_MODE_TILED, TiledTensorCore = QLB_MODE_TILED_TC };

    // cpu_openmp_engine.hpp:65-80
    explicit CUDAEngine(uint32_t num_qubits, std::optional<uint64_t> seed = std::nullopt,
                        std::size_t reserve_meas = 0) {
        b200_detail::check(
            qlb_engine_create(&h_, num_qubits, seed.has_value(), seed.value_or(0), reserve_meas));
    }
    // cpu_openmp_engine.hpp:87-102
    explicit CUDAEngine(std::span<const std::complex<double>> initial_state,
                        std::optional<uint64_t> seed = std::nullopt, std::size_t reserve_meas = 0) {
        b200_detail::check(qlb_engine_create_from_amplitudes(&h_, reinterpret_cast<const double*>(initial_state.data()),
                                                             initial_state.size(), seed.has_value(), seed.value_or(0),
                                                             reserve_meas));
    }
    // cpu_openmp_engine.hpp:105-107 (the device buffer moves, no copy)
    explicit CUDAEngine(CUDAStateVector&& sv) { b200_detail::check(qlb_engine_create_from_state(&h_, sv.handle())); }

    ~CUDAEngine() override {
        if (h_) qlb_engine_destroy(h_);
    }
    CUDAEngine(CUDAEngine&& o) noexcept
        : h_(std::exchange(o.h_, nullptr)), mirror_(std::move(o.mirror_)), meas_(std::move(o.meas_)) {}
    CUDAEngine& operator=(CUDAEngine&& o) noexcept {
        std::swap(h_, o.h_);
        mirror_.swap(o.mirror_);
        meas_.swap(o.meas_);
        return *this;
    }

    // cpu_openmp_engine.hpp:110-112, 245-247; release_state_vector as the
    // reference README describes it.
    void set_state_vector(CUDAStateVector&& sv) { b200_detail::check(qlb_engine_set_state_vector(h_, sv.handle())); }
    [[nodiscard]] CUDAStateVector extract_state_vector() && {
        CUDAStateVector out;
        b200_detail::check(qlb_engine_extract_state_vector(h_, out.handle()));
        return out;
    }
    [[nodiscard]] std::unique_ptr<StateVector> release_state_vector() {
        auto out = std::make_unique<CUDAStateVector>();
        b200_detail::check(qlb_engine_extract_state_vector(h_, out->handle()));
        return out;
    }

    // ExecutionEngine interface
    void reset() override { b200_detail::check(qlb_engine_reset(h_)); }
    void reset(std::span<const std::complex<double>> initial_state) override {
        b200_detail::check(
            qlb_engine_reset_to(h_, reinterpret_cast<const double*>(initial_state.data()), initial_state.size()));
    }
    void set_seed(uint64_t seed) override { b200_detail::check(qlb_engine_set_seed(h_, seed)); }
    void reserve_measurements(std::size_t count) override {
        b200_detail::check(qlb_engine_reserve_measurements(h_, count));
    }
    [[nodiscard]] const std::vector<uint8_t>& measurements() const override {
        const uint8_t* p = nullptr;
        uint64_t n = 0;
        b200_detail::check(qlb_engine_measurements(h_, &p, &n));
        meas_.assign(p, p + n);
        return meas_;
    }
    void execute(std::span<const GateInstr> program, const UnitaryPool& pool) override {
        const qlb_pool_view pv = b200_detail::pool_view(pool);
        b200_detail::check(
            qlb_engine_execute(h_, reinterpret_cast<const qlb_gate_instr*>(program.data()), program.size(), &pv));
    }
    // A host mirror of the device state (D2H + widen), valid until the next
    // mutating call -- the reference returns a zero-copy span instead.
    [[nodiscard]] std::span<const std::complex<double>> state() const override {
        uint32_t n = 0;
        b200_detail::check(qlb_engine_num_qubits(h_, &n));
        mirror_.resize(std::size_t{1} << n);
        b200_detail::check(qlb_engine_state(h_, reinterpret_cast<double*>(mirror_.data()), mirror_.size()));
        return mirror_;
    }
    [[nodiscard]] uint32_t num_qubits() const override {
        uint32_t n = 0;
        b200_detail::check(qlb_engine_num_qubits(h_, &n));
        return n;
    }

    // B200 extras
    void set_mode(Mode m) { b200_detail::check(qlb_engine_set_mode(h_, static_cast<int>(m))); }
    void set_physical_global_swap(bool on) {
        b200_detail::check(qlb_engine_set_option(h_, QLB_OPT_PHYSICAL_GLOBAL_SWAP, on ? 1 : 0));
    }
    [[nodiscard]] std::vector<double> expect_z() const {
        std::vector<double> out(num_qubits());
        b200_detail::check(qlb_engine_expect_z(h_, out.data(), static_cast<uint32_t>(out.size())));
        return out;
    }
    [[nodiscard]] double norm_sq() const {
        double v = 0.0;
        b200_detail::check(qlb_engine_norm_sq(h_, &v));
        return v;
    }
    [[nodiscard]] std::vector<uint64_t> sample(uint64_t seed, uint64_t shots) const {
        std::vector<uint64_t> out(shots);
        b200_detail::check(qlb_engine_sample(h_, seed, shots, out.data()));
        return out;
    }
    [[nodiscard]] qlb_engine_t handle() const noexcept { return h_; }

private:
    qlb_engine_t h_ = nullptr;
    mutable std::vector<std::complex<double>> mirror_;
    mutable std::vector<uint8_t> meas_;
};

}  // namespace qlassical::backend

// C++ drop-in tests: the reference's own backend / frontend / integration
// test cases (tests/backend/test_engine_kernels.cpp, test_engine_measure.cpp,
// test_state_vector.cpp, tests/frontend/test_circuit_runner.cpp,
// tests/integration/algos_no_optimization.cpp) restated against
// CUDAEngine / CUDAStateVector / GPUCircuitRunner, plus differential runs
// against the reference CPUOpenMPEngine compiled into this binary.
//
// Build: tests/cpp/Makefile (needs the reference include tree at build time
// only).  Run: tests/cpp/_bin/test_cuda_engine [filter]; exit status 0 when
// every check passes.  Needs a CUDA device.
#include <qlassical_b200/cuda_engine.hpp>
#include <qlassical_b200/gpu_runner.hpp>

#include <frontend/circuit_runner.hpp>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <functional>
#include <random>
#include <string>
#include <vector>

using namespace qlassical;
using namespace qlassical::backend;
using cd = std::complex<double>;

namespace {

int g_checks = 0, g_failures = 0;
const char* g_test = "";

#define CHECK(cond)                                                                              \
    do {                                                                                         \
        ++g_checks;                                                                              \
        if (!(cond)) {                                                                           \
            ++g_failures;                                                                        \
            std::fprintf(stderr, "[%s] %s:%d: CHECK(%s) failed\n", g_test, __FILE__, __LINE__, #cond); \
        }                                                                                        \
    } while (0)

#define CHECK_NEAR(a, b, tol)                                                                    \
    do {                                                                                         \
        ++g_checks;                                                                              \
        const double va_ = (a), vb_ = (b);                                                       \
        if (!(std::abs(va_ - vb_) <= (tol))) {                                                   \
            ++g_failures;                                                                        \
            std::fprintf(stderr, "[%s] %s:%d: %s = %.9g, expected %.9g (tol %g)\n", g_test, __FILE__, \
                         __LINE__, #a, va_, vb_, static_cast<double>(tol));                      \
        }                                                                                        \
    } while (0)

#define CHECK_THROWS_AS(expr, T)                                                                 \
    do {                                                                                         \
        ++g_checks;                                                                              \
        bool ok_ = false;                                                                        \
        try {                                                                                    \
            (void)(expr);                                                                        \
        } catch (const T&) {                                                                     \
            ok_ = true;                                                                          \
        } catch (...) {                                                                          \
        }                                                                                        \
        if (!ok_) {                                                                              \
            ++g_failures;                                                                        \
            std::fprintf(stderr, "[%s] %s:%d: %s did not throw %s\n", g_test, __FILE__, __LINE__, #expr, #T); \
        }                                                                                        \
    } while (0)

struct TestCase {
    const char* name;
    void (*fn)();
};
std::vector<TestCase>& registry() {
    static std::vector<TestCase> r;
    return r;
}
struct Reg {
    Reg(const char* n, void (*f)()) { registry().push_back({n, f}); }
};
#define TEST(name)                        \
    static void name();                   \
    static const Reg reg_##name(#name, name); \
    static void name()

// complex64 storage: amplitudes carry ~1e-7 relative error per gate.
constexpr double kAmpTol = 2e-6;
constexpr double kInfidelityTol = 1e-6;

const CUDAEngine::Mode kModes[] = {CUDAEngine::Mode::Plain, CUDAEngine::Mode::Tiled,
                                   CUDAEngine::Mode::TiledTensorCore};
const char* mode_name(CUDAEngine::Mode m) {
    switch (m) {
    case CUDAEngine::Mode::Plain: return "plain";
    case CUDAEngine::Mode::Tiled: return "tiled";
    default: return "tiled_tc";
    }
}

double infidelity(std::span<const cd> a, std::span<const cd> b) {
    cd ip = 0.0;
    double na = 0.0, nb = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) {
        ip += std::conj(a[i]) * b[i];
        na += std::norm(a[i]);
        nb += std::norm(b[i]);
    }
    return 1.0 - std::norm(ip) / (na * nb);
}
double max_abs_diff(std::span<const cd> a, std::span<const cd> b) {
    double m = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) m = std::max(m, std::abs(a[i] - b[i]));
    return m;
}

// GateInstr builder of the reference tests (test_engine_measure.cpp:21-43).
GateInstr make_gate(GateType t, uint8_t q0 = 255, uint8_t q1 = 255, uint8_t q2 = 255, float param = 0.0f,
                    uint32_t mat_idx = 0) {
    GateInstr g{};
    g.type = t;
    uint8_t arity = 0;
    g.qubits[0] = g.qubits[1] = g.qubits[2] = g.qubits[3] = 255;
    if (q0 != 255) { g.qubits[0] = q0; arity = 1; }
    if (q1 != 255) { g.qubits[1] = q1; arity = 2; }
    if (q2 != 255) { g.qubits[2] = q2; arity = 3; }
    g.flags_arity = arity;
    if (t == GateType::RX || t == GateType::RY || t == GateType::RZ) g.payload.param = param;
    else if (t == GateType::UNITARY || t == GateType::FUSED_BLOCK) g.payload.matrix_idx = mat_idx;
    return g;
}

std::vector<cd> random_state(uint32_t n, uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> g;
    std::vector<cd> v(std::size_t{1} << n);
    double s = 0.0;
    for (auto& a : v) {
        a = cd(g(rng), g(rng));
        s += std::norm(a);
    }
    for (auto& a : v) a /= std::sqrt(s);
    return v;
}

std::vector<cd> random_unitary(uint32_t k, std::mt19937_64& rng) {
    const std::size_t d = std::size_t{1} << k;
    std::normal_distribution<double> g;
    std::vector<cd> m(d * d);
    for (auto& a : m) a = cd(g(rng), g(rng));
    // Gram-Schmidt on the rows.
    for (std::size_t r = 0; r < d; ++r) {
        for (std::size_t p = 0; p < r; ++p) {
            cd ip = 0.0;
            for (std::size_t c = 0; c < d; ++c) ip += std::conj(m[p * d + c]) * m[r * d + c];
            for (std::size_t c = 0; c < d; ++c) m[r * d + c] -= ip * m[p * d + c];
        }
        double nn = 0.0;
        for (std::size_t c = 0; c < d; ++c) nn += std::norm(m[r * d + c]);
        nn = std::sqrt(nn);
        for (std::size_t c = 0; c < d; ++c) m[r * d + c] /= nn;
    }
    return m;
}

// A random circuit over the reference's whole gate set.
IRModule random_module(uint32_t n, std::size_t gates, uint64_t seed, bool with_unitaries = true) {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> ang(-M_PI, M_PI);
    QuantumCircuit qc(n, gates);
    auto pick = [&](uint32_t k) {
        std::vector<int16_t> q(n);
        for (uint32_t i = 0; i < n; ++i) q[i] = static_cast<int16_t>(i);
        std::shuffle(q.begin(), q.end(), rng);
        q.resize(k);
        return q;
    };
    for (std::size_t g = 0; g < gates; ++g) {
        const int kind = static_cast<int>(rng() % (with_unitaries ? 13 : 12));
        if (kind <= 4) {
            const auto q = pick(1)[0];
            switch (kind) {
            case 0: qc.h(q); break;
            case 1: qc.x(q); break;
            case 2: qc.y(q); break;
            case 3: qc.z(q); break;
            default: qc.s(q); break;
            }
        } else if (kind <= 7) {
            const auto q = pick(1)[0];
            const double a = ang(rng);
            if (kind == 5) qc.rx(q, a);
            else if (kind == 6) qc.ry(q, a);
            else qc.rz(q, a);
        } else if (kind <= 9 && n >= 2) {
            const auto q = pick(2);
            if (kind == 8) qc.cx(q[0], q[1]);
            else qc.swap(q[0], q[1]);
        } else if (kind <= 11 && n >= 3) {
            const auto q = pick(3);
            if (kind == 10) qc.ccx(q[0], q[1], q[2]);
            else qc.cswap(q[0], q[1], q[2]);
        } else if (kind == 12) {
            const uint32_t k = 1 + static_cast<uint32_t>(rng() % std::min<uint32_t>(4, n));
            const auto q = pick(k);
            const auto u = random_unitary(k, rng);
            qc.unitary(q, u);
        }
    }
    return std::move(qc).release();
}

std::vector<cd> cpu_state(const IRModule& m, std::span<const cd> init = {}) {
    auto engine = init.empty() ? CPUOpenMPEngine(m.num_qubits) : CPUOpenMPEngine(init);
    engine.execute(m);
    auto s = engine.state();
    return {s.begin(), s.end()};
}

void check_against_cpu(const IRModule& m, std::span<const cd> init = {}) {
    const auto ref = cpu_state(m, init);
    for (auto mode : kModes) {
        auto engine = init.empty() ? CUDAEngine(m.num_qubits) : CUDAEngine(init);
        engine.set_mode(mode);
        engine.execute(m);
        const auto got = engine.state();
        const double inf = infidelity(ref, got);
        const double mad = max_abs_diff(ref, got);
        if (!(inf <= kInfidelityTol && mad <= 1e-4))
            std::fprintf(stderr, "[%s] mode %s n=%u gates=%zu: infidelity %.3g max|diff| %.3g\n", g_test,
                         mode_name(mode), m.num_qubits, m.gate_stream.size(), inf, mad);
        CHECK(inf <= kInfidelityTol);
        CHECK(mad <= 1e-4);
    }
}

// ---------------------------------------------------------------------------
// tests/backend/test_engine_kernels.cpp
// ---------------------------------------------------------------------------

TEST(single_qubit_gate_kernels) {
    // Every 1-qubit gate on every qubit of a random 3-qubit state.
    const GateType types[] = {GateType::H, GateType::X, GateType::Y, GateType::Z, GateType::S};
    for (auto t : types)
        for (uint8_t q = 0; q < 3; ++q) {
            IRModule m(3);
            m.gate_stream.push_back(make_gate(t, q));
            check_against_cpu(m, random_state(3, 7 + q));
        }
    // X|0> = |1>, H|0> = |+> (test_engine_kernels.cpp:48-93)
    CUDAEngine e(1);
    UnitaryPool pool;
    std::vector<GateInstr> prog = {make_gate(GateType::X, 0)};
    e.execute(prog, pool);
    CHECK_NEAR(e.state()[1].real(), 1.0, kAmpTol);
    e.reset();
    prog = {make_gate(GateType::H, 0)};
    e.execute(prog, pool);
    CHECK_NEAR(e.state()[0].real(), M_SQRT1_2, kAmpTol);
    CHECK_NEAR(e.state()[1].real(), M_SQRT1_2, kAmpTol);
    // S|+> = (|0> + i|1>)/sqrt2
    prog = {make_gate(GateType::S, 0)};
    e.execute(prog, pool);
    CHECK_NEAR(e.state()[1].imag(), M_SQRT1_2, kAmpTol);
}

TEST(parametric_single_qubit_kernels) {
    const float angles[] = {0.0f, 0.3f, 1.5707964f, 3.1415927f, -2.2f};
    for (auto t : {GateType::RX, GateType::RY, GateType::RZ})
        for (float a : angles)
            for (uint8_t q = 0; q < 2; ++q) {
                IRModule m(2);
                m.gate_stream.push_back(make_gate(t, q, 255, 255, a));
                check_against_cpu(m, random_state(2, 11));
            }
    // RX(pi)|0> = -i|1>
    CUDAEngine e(1);
    UnitaryPool pool;
    std::vector<GateInstr> prog = {make_gate(GateType::RX, 0, 255, 255, static_cast<float>(M_PI))};
    e.execute(prog, pool);
    CHECK_NEAR(std::abs(e.state()[0]), 0.0, kAmpTol);
    CHECK_NEAR(e.state()[1].imag(), -1.0, kAmpTol);
}

TEST(multi_qubit_kernels_routing_stress) {
    // CX, SWAP, CCX, CSWAP on every ordered choice of qubits in a 4-qubit register.
    for (uint8_t a = 0; a < 4; ++a)
        for (uint8_t b = 0; b < 4; ++b) {
            if (a == b) continue;
            IRModule m(4);
            m.gate_stream.push_back(make_gate(GateType::CX, a, b));
            m.gate_stream.push_back(make_gate(GateType::SWAP, b, a));
            check_against_cpu(m, random_state(4, 100 + 4 * a + b));
            for (uint8_t c = 0; c < 4; ++c) {
                if (c == a || c == b) continue;
                IRModule m3(4);
                m3.gate_stream.push_back(make_gate(GateType::CCX, a, b, c));
                m3.gate_stream.push_back(make_gate(GateType::CSWAP, c, a, b));
                check_against_cpu(m3, random_state(4, 200 + 16 * a + 4 * b + c));
            }
        }
    // Toffoli truth table on |110> (q0 = q1 = 1) -> |111>
    CUDAEngine e(3);
    UnitaryPool pool;
    std::vector<GateInstr> prog = {make_gate(GateType::X, 0), make_gate(GateType::X, 1),
                                   make_gate(GateType::CCX, 0, 1, 2)};
    e.execute(prog, pool);
    CHECK_NEAR(e.state()[7].real(), 1.0, kAmpTol);
}

TEST(custom_unitary_gather_scatter) {
    std::mt19937_64 rng(5);
    for (uint32_t k = 1; k <= 4; ++k)
        for (int trial = 0; trial < 4; ++trial) {
            IRModule m(6);
            std::vector<int16_t> q = {0, 1, 2, 3, 4, 5};
            std::shuffle(q.begin(), q.end(), rng);
            q.resize(k);
            const auto u = random_unitary(k, rng);
            const uint32_t idx = m.unitary_pool.store(u, static_cast<uint8_t>(k));
            GateInstr g{};
            g.type = trial % 2 ? GateType::FUSED_BLOCK : GateType::UNITARY;
            g.set_arity(static_cast<uint8_t>(k));
            g.payload.matrix_idx = idx;
            for (uint32_t i = 0; i < 4; ++i) g.qubits[i] = i < k ? static_cast<uint8_t>(q[i]) : 255;
            m.gate_stream.push_back(g);
            check_against_cpu(m, random_state(6, 300 + 10 * k + trial));
        }
}

TEST(phase_kickback_circuit) {
    // X(1) H(0) H(1) CX(0,1) H(0): the phase kicks back onto q0 -> |11>.
    CUDAEngine e(2);
    QuantumCircuit qc(2);
    qc.x(1).h(0).h(1).cx(0, 1).h(0);
    e.execute(qc.release());
    const auto s = e.state();
    CHECK_NEAR(std::norm(s[1]) + std::norm(s[3]), 1.0, 1e-6);
}

// ---------------------------------------------------------------------------
// tests/backend/test_engine_measure.cpp
// ---------------------------------------------------------------------------

TEST(born_rule_and_seeded_outcomes) {
    UnitaryPool pool;
    std::vector<GateInstr> prog = {make_gate(GateType::H, 0), make_gate(GateType::MEASURE, 0)};
    for (uint64_t seed : {42ull, 1ull, 7ull, 12345ull}) {
        CPUOpenMPEngine cpu(1, seed);
        CUDAEngine gpu(1, seed);
        cpu.execute(prog, pool);
        gpu.execute(prog, pool);
        CHECK(gpu.measurements().size() == 1);
        CHECK(gpu.measurements() == cpu.measurements());
        const auto s = gpu.state();
        const uint8_t out = gpu.measurements()[0];
        CHECK_NEAR(std::abs(s[out]), 1.0, kAmpTol);
        CHECK_NEAR(std::abs(s[out ^ 1]), 0.0, kAmpTol);
    }
    // Reset clears the record and restores |0>.
    CUDAEngine e(1, 42);
    e.execute(prog, pool);
    e.reset();
    CHECK(e.measurements().empty());
    CHECK_NEAR(e.state()[0].real(), 1.0, 0.0);
    // Statistics over many seeds: both outcomes of H|0> occur.
    int ones = 0;
    for (uint64_t seed = 0; seed < 200; ++seed) {
        e.reset();
        e.set_seed(seed);
        e.execute(prog, pool);
        ones += e.measurements()[0];
    }
    CHECK(ones > 60 && ones < 140);
}

TEST(bell_state_multiple_measurements) {
    UnitaryPool pool;
    std::vector<GateInstr> prog = {make_gate(GateType::H, 0), make_gate(GateType::CX, 0, 1),
                                   make_gate(GateType::MEASURE, 0), make_gate(GateType::MEASURE, 1)};
    for (uint64_t seed = 0; seed < 32; ++seed) {
        CPUOpenMPEngine cpu(2, seed);
        CUDAEngine gpu(2, seed);
        cpu.execute(prog, pool);
        gpu.execute(prog, pool);
        const auto& ms = gpu.measurements();
        CHECK(ms.size() == 2);
        CHECK(ms[0] == ms[1]);
        CHECK(ms == cpu.measurements());
    }
}

// ---------------------------------------------------------------------------
// tests/backend/test_state_vector.cpp
// ---------------------------------------------------------------------------

TEST(state_vector_initialization_and_reset) {
    CUDAStateVector sv;
    CHECK(sv.empty());
    CHECK(sv.num_qubits() == 0);
    sv.initialize(3);
    CHECK(sv.num_qubits() == 3);
    CHECK(sv.dimension() == 8);
    auto a = sv.amplitudes();
    CHECK_NEAR(a[0].real(), 1.0, 0.0);
    for (std::size_t i = 1; i < 8; ++i) CHECK_NEAR(std::abs(a[i]), 0.0, 0.0);
    const auto init = random_state(3, 9);
    sv.initialize(init);
    a = sv.amplitudes();
    CHECK(max_abs_diff(a, init) < 1e-7);
    // Not a power of two / not normalised / empty -> invalid_argument.
    std::vector<cd> bad3(3, cd(1.0 / std::sqrt(3.0), 0.0));
    CHECK_THROWS_AS(sv.initialize(bad3), std::invalid_argument);
    std::vector<cd> unnorm(4, cd(1.0, 0.0));
    CHECK_THROWS_AS(sv.initialize(unnorm), std::invalid_argument);
    CHECK_THROWS_AS(sv.initialize(std::span<const cd>{}), std::invalid_argument);
    // Engine reset to an explicit state; like CPUOpenMPEngine::reset(span)
    // (cpu_openmp_engine.hpp:125-128) it re-sizes the register.
    CUDAEngine e(3);
    e.reset(init);
    CHECK(max_abs_diff(e.state(), init) < 1e-7);
    const auto two = random_state(2, 3);
    e.reset(two);
    CHECK(e.num_qubits() == 2);
    CHECK(max_abs_diff(e.state(), two) < 1e-7);
    CHECK_THROWS_AS(e.reset(unnorm), std::invalid_argument);
    // Moving the device buffer between engines keeps the amplitudes.
    CUDAEngine a1(init);
    CUDAStateVector moved = std::move(a1).extract_state_vector();
    CHECK(moved.num_qubits() == 3);
    CUDAEngine a2(std::move(moved));
    CHECK(max_abs_diff(a2.state(), init) < 1e-7);
    auto released = a2.release_state_vector();
    CHECK(released->num_qubits() == 3);
}

// ---------------------------------------------------------------------------
// tests/integration/algos_no_optimization.cpp
// ---------------------------------------------------------------------------

TEST(deutsch_algorithm) {
    // Balanced oracle f(x) = x (CX) -> q0 measures 1; constant oracle -> 0.
    for (int balanced = 0; balanced < 2; ++balanced) {
        CUDAEngine e(2, 42ull, 1);
        QuantumCircuit qc(2);
        qc.x(1).h(0).h(1);
        if (balanced) qc.cx(0, 1);
        qc.h(0).measure(0);
        e.execute(qc.release());
        CHECK(e.measurements().size() == 1);
        CHECK(e.measurements()[0] == balanced);
    }
}

TEST(quantum_teleportation) {
    const cd alpha(1.0 / std::sqrt(3.0), 0.0), beta(0.0, std::sqrt(2.0 / 3.0));
    for (uint64_t seed = 0; seed < 16; ++seed) {
        std::vector<cd> init(8, cd(0.0, 0.0));
        init[0] = alpha;
        init[1] = beta;
        CUDAEngine engine(init, seed, 2);
        QuantumCircuit alice(3);
        alice.h(1).cx(1, 2).cx(0, 1).h(0).measure(0).measure(1);
        engine.execute(alice.release());
        const auto ms = engine.measurements();
        CHECK(ms.size() == 2);
        const uint8_t m0 = ms[0], m1 = ms[1];
        QuantumCircuit bob(3);
        if (m1) bob.x(2);
        if (m0) bob.z(2);
        engine.execute(bob.release());
        const auto s = engine.state();
        const std::size_t i0 = (std::size_t{m1} << 1) | m0, i1 = 4 | i0;
        CHECK_NEAR(std::abs(s[i0] - alpha), 0.0, kAmpTol);
        CHECK_NEAR(std::abs(s[i1] - beta), 0.0, kAmpTol);
        // Same outcomes as the reference engine for the same seed.
        std::vector<cd> init2(8, cd(0.0, 0.0));
        init2[0] = alpha;
        init2[1] = beta;
        CPUOpenMPEngine cpu(init2, seed, 2);
        QuantumCircuit alice2(3);
        alice2.h(1).cx(1, 2).cx(0, 1).h(0).measure(0).measure(1);
        cpu.execute(alice2.release());
        CHECK(cpu.measurements() == ms);
    }
}

// ---------------------------------------------------------------------------
// tests/frontend/test_circuit_runner.cpp, Backend::GPU
// ---------------------------------------------------------------------------

TEST(gpu_runner_construction_and_guards) {
    CHECK_THROWS_AS(GPUCircuitRunner(std::shared_ptr<QuantumCircuit>{}), std::invalid_argument);
    CHECK_THROWS_AS(GPUCircuitRunner(std::vector<std::shared_ptr<QuantumCircuit>>{}), std::invalid_argument);
    CHECK_THROWS_AS(GPUCircuitRunner(std::vector<std::shared_ptr<QuantumCircuit>>{
                        std::make_shared<QuantumCircuit>(1), nullptr}),
                    std::invalid_argument);
    GPUCircuitRunner r(std::make_shared<QuantumCircuit>(2));
    CHECK_THROWS_AS(r.state(), std::runtime_error);
    CHECK_THROWS_AS(r.num_qubits(), std::runtime_error);
    CHECK(r.backend() == Backend::GPU);
    CHECK(r.num_blocks() == 1);
    r.run();
    CHECK(r.num_qubits() == 2);
    CHECK_NEAR(r.state()[0].real(), 1.0, 0.0);
}

TEST(gpu_runner_multiblock_continuity) {
    {
        auto b1 = std::make_shared<QuantumCircuit>(2);
        b1->h(0);
        auto b2 = std::make_shared<QuantumCircuit>(2);
        b2->x(1);
        auto b3 = std::make_shared<QuantumCircuit>(2);
        b3->h(0);
        GPUCircuitRunner r(std::vector<std::shared_ptr<QuantumCircuit>>{b1, b2, b3});
        r.run();
        CHECK_NEAR(r.state()[2].real(), 1.0, kAmpTol);
    }
    {
        auto b1 = std::make_shared<QuantumCircuit>(1);
        b1->x(0);
        auto b2 = std::make_shared<QuantumCircuit>(1);
        auto b3 = std::make_shared<QuantumCircuit>(1);
        b3->h(0);
        GPUCircuitRunner r(std::vector<std::shared_ptr<QuantumCircuit>>{b1, b2, b3});
        r.run();
        CHECK_NEAR(r.state()[0].real(), M_SQRT1_2, kAmpTol);
        CHECK_NEAR(r.state()[1].real(), -M_SQRT1_2, kAmpTol);
    }
    {
        std::vector<std::shared_ptr<QuantumCircuit>> blocks;
        for (int i = 0; i < 6; ++i) {
            auto b = std::make_shared<QuantumCircuit>(1);
            b->x(0);
            blocks.push_back(b);
        }
        GPUCircuitRunner r(blocks);
        r.run();
        CHECK_NEAR(r.state()[0].real(), 1.0, kAmpTol);
    }
    {
        auto b1 = std::make_shared<QuantumCircuit>(2);
        auto b2 = std::make_shared<QuantumCircuit>(3);
        GPUCircuitRunner r(std::vector<std::shared_ptr<QuantumCircuit>>{b1, b2});
        CHECK_THROWS_AS(r.run(), std::invalid_argument);
    }
    {
        // Uniform superposition across 6 qubits (64 states).
        auto b = std::make_shared<QuantumCircuit>(6);
        for (int q = 0; q < 6; ++q) b->h(static_cast<int16_t>(q));
        GPUCircuitRunner r(b);
        r.run();
        for (auto a : r.state()) CHECK_NEAR(a.real(), 0.125, kAmpTol);
    }
}

TEST(gpu_runner_matches_cpu_runner_on_random_blocks) {
    // Three random 16-qubit blocks through GPUCircuitRunner (GPU fusion and
    // windowing) versus the reference CircuitRunner on CPU_OPENMP.
    std::vector<std::shared_ptr<QuantumCircuit>> gpu_blocks, cpu_blocks;
    for (uint64_t b = 0; b < 3; ++b) {
        for (auto* v : {&gpu_blocks, &cpu_blocks}) {
            std::mt19937_64 rng(1000 + b);
            std::uniform_real_distribution<double> ang(-M_PI, M_PI);
            auto qc = std::make_shared<QuantumCircuit>(16);
            for (int g = 0; g < 120; ++g) {
                const int16_t q = static_cast<int16_t>(rng() % 16);
                const int16_t r = static_cast<int16_t>((q + 1 + rng() % 15) % 16);
                switch (rng() % 6) {
                case 0: qc->h(q); break;
                case 1: qc->rx(q, ang(rng)); break;
                case 2: qc->ry(q, ang(rng)); break;
                case 3: qc->rz(q, ang(rng)); break;
                case 4: qc->cx(q, r); break;
                default: qc->swap(q, r); break;
                }
            }
            v->push_back(qc);
        }
    }
    middleware::TranspilerConfig cfg;
    cfg.enable_hw_awareness = false;  // the CPU reference executes GLOBAL_SWAP as a no-op
    GPUCircuitRunner gr(gpu_blocks, cfg);
    gr.run();
    CircuitRunner cr(cpu_blocks, Backend::CPU_OPENMP, cfg);
    cr.run();
    const double inf = infidelity(cr.state(), gr.state());
    CHECK(inf <= kInfidelityTol);
    CHECK(max_abs_diff(cr.state(), gr.state()) < 1e-4);
}

TEST(transpile_gpu_config_and_custom_cost_model) {
    // A windowing cost model that never swaps, and one that always proposes
    // the first pair it can: both transpiled programs must give the same
    // state as the untranspiled module.
    struct Never : middleware::WindowingCostModel {
        std::optional<std::pair<uint16_t, uint16_t>> evaluate_swap(std::span<const uint32_t>,
                                                                  std::span<const uint16_t>,
                                                                  std::span<const uint16_t>) const override {
            return std::nullopt;
        }
        uint16_t get_k_safe() const override { return 4; }
    };
    struct Greedy : middleware::WindowingCostModel {
        std::optional<std::pair<uint16_t, uint16_t>> evaluate_swap(std::span<const uint32_t> f,
                                                                  std::span<const uint16_t> l2p,
                                                                  std::span<const uint16_t> p2l) const override {
            // hottest logical qubit outside the safe zone <-> coldest inside
            int hot = -1, cold = -1;
            for (uint16_t l = 0; l < f.size(); ++l)
                if (l2p[l] >= 4 && f[l] > 0 && (hot < 0 || f[l] > f[hot])) hot = l;
            for (uint16_t p = 0; p < 4 && p < p2l.size(); ++p)
                if (cold < 0 || f[p2l[p]] < f[cold]) cold = p2l[p];
            if (hot < 0 || cold < 0 || f[hot] <= f[cold]) return std::nullopt;
            return std::make_pair(static_cast<uint16_t>(hot), static_cast<uint16_t>(cold));
        }
        uint16_t get_k_safe() const override { return 4; }
    };
    const IRModule base = random_module(9, 200, 77, false);
    const auto ref = cpu_state(base);
    auto run_with = [&](const middleware::TranspilerConfig& cfg) {
        IRModule m(base.num_qubits);
        m.gate_stream = base.gate_stream;
        m.unitary_pool.data = base.unitary_pool.data;
        m.unitary_pool.metadata = base.unitary_pool.metadata;
        middleware::transpile_gpu(m, cfg);
        CUDAEngine e(m.num_qubits);
        e.execute(m);
        const auto got = e.state();
        CHECK(infidelity(ref, got) <= kInfidelityTol);
        return m.gate_stream.size();
    };
    middleware::TranspilerConfig cfg;
    const std::size_t fused = run_with(cfg);
    CHECK(fused < base.gate_stream.size());
    cfg.enable_gate_fusion = false;
    run_with(cfg);
    middleware::TranspilerConfig never;
    never.set_cost_model(std::make_shared<Never>());
    run_with(never);
    middleware::TranspilerConfig greedy;
    greedy.set_cost_model(std::make_shared<Greedy>());
    run_with(greedy);
    middleware::TranspilerConfig bad;
    bad.cost_model_type = middleware::CostModelType::CUSTOM;
    IRModule m2(2);
    CHECK_THROWS_AS(middleware::transpile_gpu(m2, bad), std::invalid_argument);
    // The GPU topology reports the tile width through the reference formula.
    middleware::GPUTopology topo;
    CHECK(topo.get_safe_qubit_limit() == topo.tile_qubits());
}

// ---------------------------------------------------------------------------
// Differential: random circuits over the whole gate set
// ---------------------------------------------------------------------------

TEST(random_circuits_all_modes) {
    for (uint32_t n : {1u, 2u, 3u, 5u, 8u, 12u, 13u, 14u, 17u, 20u}) {
        const IRModule m = random_module(n, 60 + 8 * n, 4000 + n);
        check_against_cpu(m);
    }
}

TEST(error_mapping) {
    CUDAEngine e(2);
    UnitaryPool pool;
    // Qubit index out of range -> invalid_argument; unknown gate type -> runtime_error.
    std::vector<GateInstr> bad = {make_gate(GateType::H, 5)};
    CHECK_THROWS_AS(e.execute(bad, pool), std::invalid_argument);
    GateInstr unk = make_gate(GateType::H, 0);
    unk.type = static_cast<GateType>(0x7F);
    std::vector<GateInstr> bad2 = {unk};
    CHECK_THROWS_AS(e.execute(bad2, pool), std::runtime_error);
    // Matrix index past the pool -> invalid_argument.
    std::vector<GateInstr> bad3 = {make_gate(GateType::UNITARY, 0, 255, 255, 0.0f, 3)};
    CHECK_THROWS_AS(e.execute(bad3, pool), std::invalid_argument);
}

}  // namespace

int main(int argc, char** argv) {
    const char* filter = argc > 1 ? argv[1] : nullptr;
    int run = 0;
    for (const auto& t : registry()) {
        if (filter && !std::strstr(t.name, filter)) continue;
        g_test = t.name;
        const int before = g_failures;
        try {
            t.fn();
        } catch (const std::exception& ex) {
            ++g_failures;
            std::fprintf(stderr, "[%s] unexpected exception: %s\n", t.name, ex.what());
        }
        std::printf("%-48s %s\n", t.name, g_failures == before ? "ok" : "FAILED");
        ++run;
    }
    std::printf("%d tests, %d checks, %d failures\n", run, g_checks, g_failures);
    return g_failures == 0 && run > 0 ? 0 : 1;
}

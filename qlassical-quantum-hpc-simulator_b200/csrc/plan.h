// plan.h -- a compiled program (qlb_plan): the step list of one execute()
// with every operand already in device memory.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"
#include "tile.h"

namespace qlb {

enum StepKind : uint8_t {
    STEP_PASS = 0,      // one tile-kernel launch (index = pass)
    STEP_PLAIN = 1,     // one plain instruction (instr, memory qubits)
    STEP_MEASURE = 2,   // MEASURE of memory qubit `instr.qubits[0]`
    STEP_SWAP = 3       // exchange of memory qubits instr.qubits[0..1] (data moves)
};

struct PlanStep {
    uint8_t kind;
    uint8_t features;   // STEP_PASS: the pass's kPass* bits (which kernel body it runs)
    uint32_t index;
    qlb_gate_instr instr;
    uint64_t mat_off;   // float2 offset of a dense matrix in the plan's device buffer
};

}  // namespace qlb

struct qlb_plan {
    uint32_t n = 0;
    int mode = 0;
    std::vector<qlb::PlanStep> steps;
    qlb::DeviceBuffer dev;   // [passes | phases | ops | matrices]
    const void* image = nullptr;   // the device image: dev.p, or a buffer the engine lends for one execute()
    size_t o_pass = 0, o_phase = 0, o_ops = 0, o_mat = 0;
    qlb_exec_stats stats{};
};

namespace qlb {
// What the planner needs to know about the engine.
struct PlanConfig {
    uint32_t n;
    int mode;
    int physical_global_swap;
    double tc_min_cost = 10.0;   // TILED_TC: smallest fused-run cost sent to the tensor cores
    int tc_chain = 1;            // TILED_TC: passes of tensor-core ops only run on the chain kernel
    int tile_low = kTileLow;     // memory qubits 0..tile_low-1 are in every tile (kTileLow..kTileLowMax)
};
// Host-only planning: the plan as JSON (steps, passes, phases, ops, matrices).
std::string describe_plan_json(const PlanConfig& cfg, const qlb_gate_instr* prog, uint64_t count,
                               const qlb_pool_view* pool);
// Host-only planning result (no device memory touched).
struct HostPlan {
    std::vector<PlanStep> steps;
    TileProgram prog;
    qlb_exec_stats stats{};
};
HostPlan plan_host(const PlanConfig& cfg, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool);
// Builds a plan for the engine's qubit count, mode and options.
// `image`: a device buffer to hold the plan (reused across calls, e.g. by
// execute()); nullptr: the plan owns its own.
qlb_plan* compile_plan(qlb_engine& e, const qlb_gate_instr* prog, uint64_t count, const qlb_pool_view* pool,
                       qlb::DeviceBuffer* image = nullptr);
void run_plan(qlb_engine& e, const qlb_plan& p);
}  // namespace qlb

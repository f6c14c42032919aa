// batch.cpp -- batched execution of many independent circuits (qlb_batch).
//
// Every circuit is planned on its own (tile passes, k <= 5 fusion inside
// tiles, deferred diagonals) by host threads; the plans are merged into one
// device program.  Round r applies the r-th pass of every circuit that has
// one, as ONE launch of the tile kernel over a work list of (state, pass)
// entries, so small circuits share the GPU's 148 SMs instead of each
// occupying a launch.  |0...0> set-up, all rounds and the FP64 <Z_i>
// reduction are captured once into a CUDA graph; qlb_batch_run() is one
// graph launch.  Circuits below 13 qubits run padded to one 13-qubit tile
// (the extra qubits stay |0>).  With mode -1 an autotuner times planner
// configurations -- FP32 CUDA-core tiles or tensor-core fused tiles, 3..5
// fixed low tile qubits -- on a sample of each size class (circuits of one
// padded qubit count), then picks the mode for the batch and the fixed low
// qubits per class.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "abi.h"
#include "batch.h"
#include "engine.h"
#include "kernels.h"
#include "plan.h"
#include "tile.h"

using namespace qlb;

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t{255}; }

struct BatchRound {
    size_t work_off;     // byte offset of its TileWork entries
    uint32_t n_work;
    uint64_t tiles;
    int features;
    size_t tmap_off;     // byte offset of its tile -> work-entry table (u32 per tile)
};

// One mode's device program and graph over the shared state buffer.
struct BatchProgram {
    int mode = QLB_MODE_TILED;
    DeviceBuffer dev;                // passes | phases | ops | mats | work lists
    size_t o_pass = 0, o_phase = 0, o_ops = 0, o_mat = 0;
    std::vector<BatchRound> rounds;
    uint64_t tiles = 0, passes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    float graph_ms = 0.f;
    ~BatchProgram() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

}  // namespace

struct qlb_batch {
    cudaStream_t stream = nullptr;
    uint32_t count = 0;
    std::vector<BatchState> states;
    std::vector<uint64_t> chunk_begin;     // count + 1
    uint64_t total_amps = 0, amp_updates = 0;
    DeviceBuffer state_buf, meta, partial, result, err;
    PinnedBuffer host_result, host_err;
    size_t o_states = 0, o_chunks = 0;
    std::unique_ptr<BatchProgram> prog;
    double autotune_ms[2] = {0.0, 0.0};
    double tune_seconds = 0.0, fuse_seconds = 0.0, plan_seconds = 0.0;
    std::vector<qlb_batch_tune_class> tune;
    ~qlb_batch() {
        prog.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// A planner configuration the autotuner can pick (qlb_batch_tune_class).
struct TuneCand {
    int mode;
    int tile_low;
};
TuneCand tune_candidate(int i) { return TuneCand{i < 3 ? QLB_MODE_TILED : QLB_MODE_TILED_TC, kTileLow + i % 3}; }

struct PlanJob {
    uint32_t circuit;
    int cand;
};

// Plans every job (one circuit under one candidate) on host threads.
std::vector<HostPlan> plan_jobs(const qlb_batch& b, const std::vector<PlanJob>& jobs,
                                const qlb_gate_instr* const* programs, const uint64_t* counts,
                                const qlb_pool_view* pools) {
    const size_t J = jobs.size();
    std::vector<HostPlan> plans(J);
    std::atomic<size_t> next{0};
    std::vector<std::string> errs(J);
    std::vector<int> codes(J, 0);
    auto worker = [&] {
        for (size_t j; (j = next.fetch_add(1)) < J;) {
            const uint32_t c = jobs[j].circuit;
            const TuneCand tc = tune_candidate(jobs[j].cand);
            try {
                // work lists run on the general tile kernel: no chain passes
                const PlanConfig cfg{b.states[c].eff_qubits, tc.mode, 0, 10.0, 0, tc.tile_low};
                plans[j] = plan_host(cfg, programs[c], counts[c], &pools[c]);
            } catch (const Error& e) {
                codes[j] = e.code;
                errs[j] = e.msg;
            }
        }
    };
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    nt = static_cast<unsigned>(std::min<size_t>(nt, J));
    std::vector<std::thread> th;
    for (unsigned i = 1; i < nt; ++i) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
    for (size_t j = 0; j < J; ++j)
        if (codes[j])
            fail(static_cast<qlb_status>(codes[j]), "circuit " + std::to_string(jobs[j].circuit) + ": " + errs[j]);
    return plans;
}

// Merges the plans of `members` (plans[i] belongs to members[i]) into one
// device program of rounds over the shared state buffer.
std::unique_ptr<BatchProgram> assemble(qlb_batch& b, const std::vector<uint32_t>& members,
                                       std::vector<HostPlan>& plans, int mode) {
    const size_t C = members.size();
    // merge the small arrays (passes, phases, ops: rebased); the matrix
    // images, which tensor-core ops make large (16 KB each), go to the device
    // straight from each plan
    auto P = std::make_unique<BatchProgram>();
    P->mode = mode;
    TileProgram all;
    std::vector<std::vector<uint32_t>> pass_ids(C);
    std::vector<size_t> mat_at(C);   // float2 offset of each plan's matrices
    size_t n_mats = 0;
    size_t max_passes = 0;
    for (size_t i = 0; i < C; ++i) {
        HostPlan& h = plans[i];
        for (const PlanStep& st : h.steps)
            if (st.kind != STEP_PASS)
                fail(QLB_ERR_INVALID_ARG, "circuit " + std::to_string(members[i]) +
                                              ": batched circuits may hold only gates (no MEASURE, no 6-qubit "
                                              "blocks, no physical GLOBAL_SWAP)");
        n_mats += n_mats & 1;        // each plan's matrices start on a 16-byte boundary
        const uint32_t pb = static_cast<uint32_t>(all.passes.size());
        const uint32_t phb = static_cast<uint32_t>(all.phases.size());
        const uint32_t ob = static_cast<uint32_t>(all.ops.size());
        const uint32_t mb = static_cast<uint32_t>(n_mats);
        if (n_mats + h.prog.mats.size() > 0xFFFFFFFFull) fail(QLB_ERR_OOM, "batch matrix images exceed 32-bit offsets");
        for (TilePass p : h.prog.passes) {
            p.phase_begin += phb;
            p.phase_end += phb;
            all.passes.push_back(p);
        }
        for (TilePhase ph : h.prog.phases) {
            ph.op_begin += ob;
            ph.op_end += ob;
            all.phases.push_back(ph);
        }
        for (TileOp op : h.prog.ops) {
            op.data += mb;
            all.ops.push_back(op);
        }
        mat_at[i] = n_mats;
        n_mats += h.prog.mats.size();
        for (const PlanStep& st : h.steps) pass_ids[i].push_back(pb + st.index);
        max_passes = std::max(max_passes, pass_ids[i].size());
        P->passes += pass_ids[i].size();
    }
    // rounds: the r-th pass of every circuit that has one
    std::vector<TileWork> work;
    std::vector<uint32_t> tmap;
    for (size_t r = 0; r < max_passes; ++r) {
        BatchRound R{work.size() * sizeof(TileWork), 0, 0, 0, tmap.size() * sizeof(uint32_t)};
        for (size_t i = 0; i < C; ++i) {
            if (r >= pass_ids[i].size()) continue;
            const uint32_t c = members[i];
            const uint32_t pid = pass_ids[i][r];
            work.push_back(TileWork{nullptr, R.tiles, nullptr, nullptr, nullptr, nullptr, pid, 0});
            // state pointers are filled in below, once the buffer exists
            work.back().pad = c;
            const uint64_t nt = uint64_t{1} << (b.states[c].eff_qubits - kTileQubits);
            tmap.insert(tmap.end(), nt, R.n_work);
            R.tiles += nt;
            R.n_work += 1;
            R.features |= all.passes[pid].features;
        }
        P->tiles += R.tiles;
        P->rounds.push_back(R);
    }
    // device layout: passes | phases | ops | work lists | tile maps | matrices
    P->o_pass = 0;
    P->o_phase = align256(all.passes.size() * sizeof(TilePass));
    P->o_ops = align256(P->o_phase + all.phases.size() * sizeof(TilePhase));
    const size_t o_work = align256(P->o_ops + all.ops.size() * sizeof(TileOp));
    const size_t o_tmap = align256(o_work + work.size() * sizeof(TileWork));
    P->o_mat = align256(o_tmap + tmap.size() * sizeof(uint32_t));
    const size_t total = align256(P->o_mat + n_mats * sizeof(float2));
    char* d = static_cast<char*>(P->dev.ensure(total));
    float2* base = static_cast<float2*>(b.state_buf.p);
    for (TileWork& w : work) {
        w.state = base + b.states[w.pad].offset;
        w.pad = 0;
        w.passes = reinterpret_cast<const TilePass*>(d + P->o_pass);
        w.phases = reinterpret_cast<const TilePhase*>(d + P->o_phase);
        w.ops = reinterpret_cast<const TileOp*>(d + P->o_ops);
        w.mats = reinterpret_cast<const float2*>(d + P->o_mat);
    }
    std::vector<char> h(P->o_mat);
    std::memcpy(h.data() + P->o_pass, all.passes.data(), all.passes.size() * sizeof(TilePass));
    std::memcpy(h.data() + P->o_phase, all.phases.data(), all.phases.size() * sizeof(TilePhase));
    std::memcpy(h.data() + P->o_ops, all.ops.data(), all.ops.size() * sizeof(TileOp));
    std::memcpy(h.data() + o_work, work.data(), work.size() * sizeof(TileWork));
    std::memcpy(h.data() + o_tmap, tmap.data(), tmap.size() * sizeof(uint32_t));
    for (BatchRound& R : P->rounds) {
        R.work_off += o_work;
        R.tmap_off += o_tmap;
    }
    // On the batch's stream: it does not synchronise with the legacy default
    // stream, and a cudaMemcpy from pageable memory may return before its DMA
    // has landed, so a launch on the batch's stream could read the program early.
    check_cuda(cudaMemcpyAsync(d, h.data(), h.size(), cudaMemcpyHostToDevice, b.stream), "batch program upload");
    for (size_t i = 0; i < C; ++i)
        if (!plans[i].prog.mats.empty())
            check_cuda(cudaMemcpyAsync(d + P->o_mat + mat_at[i] * sizeof(float2), plans[i].prog.mats.data(),
                                       plans[i].prog.mats.size() * sizeof(float2), cudaMemcpyHostToDevice, b.stream),
                       "batch matrix upload");
    check_cuda(cudaStreamSynchronize(b.stream), "batch program upload");
    return P;
}

void capture(qlb_batch& b, BatchProgram& P) {
    check_cuda(configure_tile_kernel(), "tile kernel attributes");
    const char* d = static_cast<const char*>(P.dev.p);
    const auto* st = reinterpret_cast<const BatchState*>(static_cast<const char*>(b.meta.p) + b.o_states);
    const auto* chunks = reinterpret_cast<const uint64_t*>(static_cast<const char*>(b.meta.p) + b.o_chunks);
    float2* base = static_cast<float2*>(b.state_buf.p);
    int* err = static_cast<int*>(b.err.p);
    cudaStream_t s = b.stream;
    check_cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = cudaMemsetAsync(base, 0, b.total_amps * sizeof(float2), s);
    if (e == cudaSuccess) e = launch_set_basis(base, st, b.count, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    for (const BatchRound& R : P.rounds) {
        if (e != cudaSuccess) break;
        e = launch_tile_work(reinterpret_cast<const TileWork*>(d + R.work_off), R.n_work, R.tiles, R.features, err, s, 0,
                             reinterpret_cast<const uint32_t*>(d + R.tmap_off));
    }
    if (e == cudaSuccess)
        e = launch_batch_expect_z(base, st, b.count, chunks, b.chunk_begin.back(), static_cast<double*>(b.partial.p),
                                  static_cast<double*>(b.result.p), kBatchStride, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b.host_result.p, b.result.p, static_cast<size_t>(b.count) * kBatchStride * sizeof(double),
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.host_err.p, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &g);
    check_cuda(e, "batch capture");
    check_cuda(ee, "end capture");
    P.graph = g;
    check_cuda(cudaGraphInstantiate(&P.exec, g, 0), "graph instantiate");
}

// Milliseconds of one run of a program's tile rounds (no set-up, no
// reductions): one warm run, then the mean of `reps` runs between events.
float time_rounds(qlb_batch& b, const BatchProgram& P, int reps) {
    check_cuda(configure_tile_kernel(), "tile kernel attributes");
    const char* d = static_cast<const char*>(P.dev.p);
    int* err = static_cast<int*>(b.err.p);
    cudaStream_t s = b.stream;
    auto rounds = [&]() -> cudaError_t {
        for (const BatchRound& R : P.rounds) {
            const cudaError_t e =
                launch_tile_work(reinterpret_cast<const TileWork*>(d + R.work_off), R.n_work, R.tiles, R.features, err,
                                 s, 0, reinterpret_cast<const uint32_t*>(d + R.tmap_off));
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    cudaEvent_t t0, t1;
    check_cuda(cudaEventCreate(&t0), "event");
    check_cuda(cudaEventCreate(&t1), "event");
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess) e = rounds();
    if (e == cudaSuccess) e = cudaEventRecord(t0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = rounds();
    if (e == cudaSuccess) e = cudaEventRecord(t1, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.host_err.p, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(t1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    check_cuda(e, "autotune rounds");
    if (*static_cast<int*>(b.host_err.p) != 0) fail(QLB_ERR_TIMEOUT, "a tile-kernel wait gave up during autotuning");
    return ms / static_cast<float>(reps);
}

// The autotuner: for each size class, plans a sample of its circuits under
// every candidate, times the sample's rounds, and returns the candidate of
// each circuit (the fastest of its class).
std::vector<int> autotune(qlb_batch& b, const qlb_gate_instr* const* programs, const uint64_t* counts,
                          const qlb_pool_view* pools) {
    constexpr uint32_t kMaxSample = 128;
    const uint64_t target_tiles = 2 * static_cast<uint64_t>(sm_count());
    std::vector<std::vector<uint32_t>> cls(kBatchMaxQubits + 1);
    for (uint32_t c = 0; c < b.count; ++c) cls[b.states[c].eff_qubits].push_back(c);
    struct Sample {
        uint32_t ne;
        std::vector<uint32_t> members;
    };
    std::vector<Sample> samples;
    std::vector<PlanJob> jobs;
    for (uint32_t ne = kBatchMinQubits; ne <= kBatchMaxQubits; ++ne) {
        if (cls[ne].empty()) continue;
        const uint64_t per = uint64_t{1} << (ne - kTileQubits);
        const uint64_t want = std::max<uint64_t>(1, (target_tiles + per - 1) / per);
        const size_t n = static_cast<size_t>(std::min<uint64_t>({want, kMaxSample, cls[ne].size()}));
        samples.push_back(Sample{ne, std::vector<uint32_t>(cls[ne].begin(), cls[ne].begin() + static_cast<long>(n))});
        for (int k = 0; k < QLB_BATCH_TUNE_CANDIDATES; ++k)
            for (uint32_t c : samples.back().members) jobs.push_back(PlanJob{c, k});
    }
    if (samples.size() > QLB_BATCH_TUNE_CLASSES) fail(QLB_ERR_INVALID_ARG, "too many size classes");
    // Candidates that cannot plan a circuit are left out of its class's
    // search; every circuit plans under candidate 0, the engines' default.
    std::vector<HostPlan> plans(jobs.size());
    std::vector<char> planned(jobs.size(), 1);
    try {
        plans = plan_jobs(b, jobs, programs, counts, pools);
    } catch (const Error&) {
        for (size_t j = 0; j < jobs.size(); ++j) {
            try {
                std::vector<PlanJob> one{jobs[j]};
                plans[j] = std::move(plan_jobs(b, one, programs, counts, pools)[0]);
            } catch (const Error&) {
                if (jobs[j].cand == 0) throw;
                planned[j] = 0;
            }
        }
    }
    // valid, uniform states for timing
    check_cuda(cudaMemsetAsync(b.state_buf.p, 0, b.total_amps * sizeof(float2), b.stream), "autotune state");
    check_cuda(launch_set_basis(static_cast<float2*>(b.state_buf.p),
                                reinterpret_cast<const BatchState*>(static_cast<const char*>(b.meta.p) + b.o_states),
                                b.count, b.stream),
               "autotune basis");
    std::vector<int> choice(b.count, 0);
    b.tune.clear();
    b.autotune_ms[0] = b.autotune_ms[1] = 0.0;
    size_t j = 0;
    for (const Sample& S : samples) {
        qlb_batch_tune_class T{};
        T.num_qubits = S.ne;
        T.circuits = static_cast<uint32_t>(cls[S.ne].size());
        T.sample = static_cast<uint32_t>(S.members.size());
        T.best = 0;
        for (int k = 0; k < QLB_BATCH_TUNE_CANDIDATES; ++k) {
            const size_t n = S.members.size();
            bool ok = true;
            for (size_t i = 0; i < n; ++i) ok = ok && planned[j + i];
            if (ok) {
                std::vector<HostPlan> part(std::make_move_iterator(plans.begin() + static_cast<long>(j)),
                                           std::make_move_iterator(plans.begin() + static_cast<long>(j + n)));
                auto P = assemble(b, S.members, part, tune_candidate(k).mode);
                T.ms[k] = time_rounds(b, *P, 3);
            } else {
                T.ms[k] = -1.f;
            }
            j += n;
        }
        b.tune.push_back(T);
    }
    // A round launches one kernel body for all its passes (the union of
    // their needs), so a tensor-core class would move every round it shares
    // onto the tensor-core body: the mode is chosen for the whole batch, by
    // the smaller projected total of the classes' best candidates in that
    // mode, and the fixed low qubits per class.
    auto best_in = [](const qlb_batch_tune_class& T, int mode_index) {
        int best = -1;
        for (int k = 3 * mode_index; k < 3 * mode_index + 3; ++k)
            if (T.ms[k] >= 0.f && (best < 0 || T.ms[k] < T.ms[best])) best = k;
        return best;
    };
    double total[2] = {0.0, 0.0};
    bool usable[2] = {true, true};
    for (const qlb_batch_tune_class& T : b.tune) {
        const double scale = static_cast<double>(T.circuits) / static_cast<double>(T.sample);
        for (int m = 0; m < 2; ++m) {
            const int k = best_in(T, m);
            if (k < 0) usable[m] = false;
            else total[m] += scale * T.ms[k];
        }
        b.autotune_ms[1] += scale * T.ms[0];
    }
    const int mode_index = usable[1] && (!usable[0] || total[1] < total[0]) ? 1 : 0;
    b.autotune_ms[0] = total[mode_index];
    for (size_t i = 0; i < b.tune.size(); ++i) {
        b.tune[i].best = best_in(b.tune[i], mode_index);
        for (uint32_t c : cls[samples[i].ne]) choice[c] = b.tune[i].best;
    }
    return choice;
}

// Plans every circuit under its candidate and assembles the batch program.
std::unique_ptr<BatchProgram> build_program(qlb_batch& b, const std::vector<int>& choice,
                                            const qlb_gate_instr* const* programs, const uint64_t* counts,
                                            const qlb_pool_view* pools) {
    std::vector<PlanJob> jobs(b.count);
    std::vector<uint32_t> members(b.count);
    int mode = tune_candidate(choice[0]).mode;
    for (uint32_t c = 0; c < b.count; ++c) {
        jobs[c] = PlanJob{c, choice[c]};
        members[c] = c;
        if (tune_candidate(choice[c]).mode != mode) mode = -1;
    }
    std::vector<HostPlan> plans = plan_jobs(b, jobs, programs, counts, pools);
    return assemble(b, members, plans, mode);
}

}  // namespace

extern "C" {

int qlb_batch_create(qlb_batch_t* out, uint32_t count, const qlb_gate_instr* const* programs, const uint64_t* counts,
                     const qlb_pool_view* pools, const uint32_t* num_qubits, int mode) {
    return qlb_batch_create_ex(out, count, programs, counts, pools, num_qubits, mode, 0);
}

int qlb_batch_create_ex(qlb_batch_t* out, uint32_t count, const qlb_gate_instr* const* programs_in,
                        const uint64_t* counts_in, const qlb_pool_view* pools_in, const uint32_t* num_qubits,
                        int mode, uint32_t fuse_qubits) {
    return guarded([&] {
        const qlb_gate_instr* const* programs = programs_in;
        const uint64_t* counts = counts_in;
        const qlb_pool_view* pools = pools_in;
        need(out, "out");
        *out = nullptr;
        if (count == 0) fail(QLB_ERR_INVALID_ARG, "empty batch");
        need(programs, "programs");
        need(counts, "counts");
        need(pools, "pools");
        need(num_qubits, "num_qubits");
        if (mode != QLB_MODE_TILED && mode != QLB_MODE_TILED_TC && mode != -1)
            fail(QLB_ERR_INVALID_ARG, "batch mode must be QLB_MODE_TILED, QLB_MODE_TILED_TC or -1 (autotune)");
        auto b = std::make_unique<qlb_batch>();
        b->count = count;
        b->states.resize(count);
        b->chunk_begin.resize(count + 1);
        uint64_t off = 0, chunks = 0;
        for (uint32_t c = 0; c < count; ++c) {
            const uint32_t n = num_qubits[c];
            if (n == 0 || n > 30) fail(QLB_ERR_INVALID_ARG, "batched circuits take 1..30 qubits");
            if (counts[c] && !programs[c]) fail(QLB_ERR_INVALID_ARG, "null program");
            const uint32_t ne = std::max(n, kBatchMinQubits);
            b->states[c] = BatchState{off, n, ne};
            b->chunk_begin[c] = chunks;
            off += uint64_t{1} << ne;
            chunks += uint64_t{1} << (ne - kBatchMinQubits);
            for (uint64_t i = 0; i < counts[c]; ++i) {
                const qlb_gate_instr& g = programs[c][i];
                if (g.type != QLB_BARRIER && g.type != QLB_MEASURE)
                    b->amp_updates += uint64_t{1} << n;
            }
        }
        b->chunk_begin[count] = chunks;
        b->total_amps = off;
        check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
        b->state_buf.ensure(off * sizeof(float2));
        b->o_states = 0;
        b->o_chunks = align256(count * sizeof(BatchState));
        const size_t meta_bytes = b->o_chunks + (count + 1) * sizeof(uint64_t);
        char* m = static_cast<char*>(b->meta.ensure(meta_bytes));
        check_cuda(cudaMemcpyAsync(m + b->o_states, b->states.data(), count * sizeof(BatchState),
                                   cudaMemcpyHostToDevice, b->stream),
                   "batch states");
        check_cuda(cudaMemcpyAsync(m + b->o_chunks, b->chunk_begin.data(), (count + 1) * sizeof(uint64_t),
                                   cudaMemcpyHostToDevice, b->stream),
                   "batch chunks");
        check_cuda(cudaStreamSynchronize(b->stream), "batch metadata upload");
        b->partial.ensure(batch_partial_doubles(chunks) * sizeof(double));
        b->result.ensure(static_cast<size_t>(count) * kBatchStride * sizeof(double));
        b->err.ensure(256);
        b->host_result.ensure(static_cast<size_t>(count) * kBatchStride * sizeof(double));
        b->host_err.ensure(sizeof(int));
        *static_cast<int*>(b->host_err.p) = 0;
        // Fusion by the GPU middle end (blocks of up to fuse_qubits, no
        // windowing), circuit by circuit on host threads; the batch is then
        // planned from the fused programs (the counts above stay the logical
        // gates').
        struct Modules {
            std::vector<qlb_module_t> m;
            ~Modules() {
                for (qlb_module_t x : m)
                    if (x) qlb_module_destroy(x);
            }
        } fused;
        std::vector<const qlb_gate_instr*> fprog;
        std::vector<uint64_t> fcount;
        std::vector<qlb_pool_view> fpool;
        if (fuse_qubits) {
            const auto tf = std::chrono::steady_clock::now();
            if (fuse_qubits > 5) fail(QLB_ERR_INVALID_ARG, "batched fusion takes blocks of at most 5 qubits");
            fused.m.assign(count, nullptr);
            fprog.assign(count, nullptr);
            fcount.assign(count, 0);
            fpool.assign(count, qlb_pool_view{nullptr, 0, nullptr, 0});
            std::vector<std::string> errs(count);
            std::atomic<uint32_t> next{0};
            auto worker = [&] {
                qlb_transpile_config tc;
                qlb_transpile_config_default(&tc);
                tc.enable_hw_awareness = 0;
                tc.max_fusion_qubits = static_cast<int>(fuse_qubits);
                for (uint32_t c; (c = next.fetch_add(1)) < count;) {
                    if (qlb_transpile_gpu(programs_in[c], counts_in[c], &pools_in[c], num_qubits[c], &tc,
                                          &fused.m[c]) != QLB_OK) {
                        errs[c] = qlb_last_error();
                        continue;
                    }
                    qlb_module_program(fused.m[c], &fprog[c], &fcount[c]);
                    qlb_module_pool(fused.m[c], &fpool[c]);
                }
            };
            unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
            nt = std::min<unsigned>(nt, count);
            std::vector<std::thread> th;
            for (unsigned i = 1; i < nt; ++i) th.emplace_back(worker);
            worker();
            for (auto& t : th) t.join();
            for (uint32_t c = 0; c < count; ++c)
                if (!errs[c].empty()) fail(QLB_ERR_INVALID_ARG, "circuit " + std::to_string(c) + " fusion: " + errs[c]);
            programs = fprog.data();
            counts = fcount.data();
            pools = fpool.data();
            b->fuse_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tf).count();
        }
        std::vector<int> choice(count, mode == QLB_MODE_TILED_TC ? 3 : 0);
        if (mode == -1) {
            const auto t0 = std::chrono::steady_clock::now();
            choice = autotune(*b, programs, counts, pools);
            b->tune_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        const auto tp = std::chrono::steady_clock::now();
        b->prog = build_program(*b, choice, programs, counts, pools);
        capture(*b, *b->prog);
        b->plan_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tp).count();
        *out = b.release();
    });
}

int qlb_batch_run(qlb_batch_t b) {
    return guarded([&] {
        need(b, "batch");
        check_cuda(cudaGraphLaunch(b->prog->exec, b->stream), "batch graph launch");
    });
}

int qlb_batch_synchronize(qlb_batch_t b) {
    return guarded([&] {
        need(b, "batch");
        check_cuda(cudaStreamSynchronize(b->stream), "batch sync");
        if (*static_cast<int*>(b->host_err.p) != 0)
            fail(QLB_ERR_TIMEOUT, "a tile-kernel wait gave up (copy or tensor-core completion)");
    });
}

int qlb_batch_expect_z(qlb_batch_t b, double* out, uint32_t stride) {
    return guarded([&] {
        need(b, "batch");
        need(out, "out");
        const double* r = static_cast<const double*>(b->host_result.p);
        for (uint32_t c = 0; c < b->count; ++c) {
            if (stride < b->states[c].num_qubits) fail(QLB_ERR_INVALID_ARG, "stride below a circuit's qubit count");
            for (uint32_t q = 0; q < b->states[c].num_qubits; ++q)
                out[static_cast<uint64_t>(c) * stride + q] = r[static_cast<uint64_t>(c) * kBatchStride + q];
        }
    });
}

int qlb_batch_state(qlb_batch_t b, uint32_t index, double* out_c128, uint64_t dim) {
    return guarded([&] {
        need(b, "batch");
        need(out_c128, "out");
        if (index >= b->count) fail(QLB_ERR_INVALID_ARG, "circuit index out of range");
        const BatchState& s = b->states[index];
        if (dim != (uint64_t{1} << s.num_qubits)) fail(QLB_ERR_INVALID_ARG, "dim must be 2^num_qubits");
        check_cuda(cudaStreamSynchronize(b->stream), "batch sync");
        std::vector<float2> h(dim);
        check_cuda(cudaMemcpy(h.data(), static_cast<float2*>(b->state_buf.p) + s.offset, dim * sizeof(float2),
                              cudaMemcpyDeviceToHost),
                   "batch state D2H");
        for (uint64_t i = 0; i < dim; ++i) {
            out_c128[2 * i] = h[i].x;
            out_c128[2 * i + 1] = h[i].y;
        }
    });
}

int qlb_batch_stats(qlb_batch_t b, qlb_batch_info* out) {
    return guarded([&] {
        need(b, "batch");
        need(out, "out");
        out->circuits = b->count;
        out->rounds = static_cast<uint32_t>(b->prog->rounds.size());
        out->mode = b->prog->mode;
        out->launches = static_cast<uint32_t>(b->prog->rounds.size()) + 4;
        out->tiles = b->prog->tiles;
        out->passes = b->prog->passes;
        out->amp_updates = b->amp_updates;
        out->state_bytes = b->total_amps * sizeof(float2);
        out->autotune_ms[0] = b->autotune_ms[0];
        out->autotune_ms[1] = b->autotune_ms[1];
        out->tune_seconds = b->tune_seconds;
        out->fuse_seconds = b->fuse_seconds;
        out->plan_seconds = b->plan_seconds;
        out->tune_classes = static_cast<uint32_t>(b->tune.size());
        for (size_t i = 0; i < b->tune.size() && i < QLB_BATCH_TUNE_CLASSES; ++i) out->tune[i] = b->tune[i];
    });
}

int qlb_batch_stream(qlb_batch_t b, void** out) {
    return guarded([&] {
        need(b, "batch");
        need(out, "out");
        *out = b->stream;
    });
}

int qlb_batch_destroy(qlb_batch_t b) {
    return guarded([&] {
        if (!b) return;
        cudaStreamSynchronize(b->stream);
        delete b;
    });
}

}  // extern "C"

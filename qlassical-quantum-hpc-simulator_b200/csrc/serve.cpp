// serve.cpp -- the serving loop (qlb_server): continuous batching of
// independent circuit requests on one GPU.
//
// A request (circuit, shots, seed) is planned on the submitting thread
// (tile passes, as the engine would).  The server thread admits queued
// requests in arrival order while their state vector, program and sampling
// scratch fit in a device arena sized from free HBM (no allocation on the
// hot path), then advances every admitted request by one pass per round:
// one tile-kernel launch over a work list of (state, program, pass)
// entries.  Requests that arrive while others run join at the next round
// boundary.  When a request's last pass has run, the same round ends with
// its FP64 <Z_i> reduction and `shots` counter-based samples; results go to
// pinned host memory and its arena blocks are released.  A request's results
// are bitwise the same whatever else shares its rounds: the tile kernel,
// the per-state reduction order and the (seed, shot)-keyed sampling do not
// depend on the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
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

// First-fit allocator over one device allocation; blocks are 256-B aligned.
class Arena {
public:
    void init(size_t bytes) {
        bytes_ = bytes & ~size_t{255};
        free_.clear();
        free_[0] = bytes_;
        used_ = 0;
    }
    bool alloc(size_t bytes, size_t& off) {
        bytes = align256(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            off = it->first;
            const size_t rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = align256(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t capacity() const { return bytes_; }
    size_t used() const { return used_; }

private:
    size_t bytes_ = 0, used_ = 0;
    std::map<size_t, size_t> free_;
};

enum ReqState { REQ_QUEUED = 0, REQ_ACTIVE = 1, REQ_DONE = 2, REQ_FAILED = 3, REQ_CANCELLED = 4 };

struct Request {
    uint64_t id = 0;
    uint32_t n = 0, neff = 0;
    uint64_t shots = 0, seed = 0;
    HostPlan plan;
    std::vector<uint32_t> pass_features;
    // device layout inside one arena block: state | program | sample scratch
    size_t block_off = 0, block_bytes = 0;
    size_t o_state = 0, o_pass = 0, o_phase = 0, o_ops = 0, o_mat = 0, o_chunk = 0, o_samples = 0;
    std::vector<char> prog_image;   // passes | phases | ops | mats, offsets relative to o_pass
    uint32_t next_pass = 0;
    bool cancel = false;            // set by qlb_server_cancel while admitted
    int status = REQ_QUEUED;
    std::string error;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> ez;
    std::vector<uint64_t> samples;
};

}  // namespace

namespace {

constexpr uint32_t kMaxWork = 4096;
constexpr uint32_t kLargeQubits = 22;    // requests of >= 22 qubits run in the large lane
constexpr uint32_t kSmallLaneCtas = 20;  // SMs left to the small lane while both lanes run

// One lane: its own stream, admitted requests and per-round buffers.
struct Lane {
    int index = 0;
    cudaStream_t stream = nullptr;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> active;
    DeviceBuffer work_dev, meta_dev, partial_dev, result_dev, err_dev;
    PinnedBuffer work_host, meta_host, result_host, err_host;
    std::thread worker;
    ~Lane() {
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

struct qlb_server {
    int device = 0;
    int mode = QLB_MODE_TILED;
    uint32_t fuse_from = 0;            // requests of >= fuse_from qubits: fused, tensor-core plans
    uint32_t max_active = 4096;
    Arena arena;
    DeviceBuffer arena_mem;
    size_t max_chunks = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    Lane lanes[2];                     // 0: small states, 1: large states
    std::unordered_map<uint64_t, std::shared_ptr<Request>> all;
    uint64_t next_id = 1;
    bool stop = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    qlb_server_info info{};
    std::string fatal;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

// Admits the lane's queued requests in order while they fit; returns how many.
uint32_t admit(qlb_server& s, Lane& L) {
    uint32_t added = 0;
    while (!L.queue.empty() && s.lanes[0].active.size() + s.lanes[1].active.size() < s.max_active) {
        auto& r = L.queue.front();
        size_t off = 0;
        if (!s.arena.alloc(r->block_bytes, off)) break;
        r->block_off = off;
        r->status = REQ_ACTIVE;
        r->t_admit = s.now();
        L.active.push_back(r);
        L.queue.pop_front();
        ++added;
    }
    return added;
}

void fail_all(qlb_server& s, const std::string& why) {
    s.fatal = why;
    for (Lane& L : s.lanes) {
        for (auto& r : L.active) {
            r->status = REQ_FAILED;
            r->error = why;
            r->t_done = s.now();
        }
        L.active.clear();
        for (auto& r : L.queue) {
            r->status = REQ_FAILED;
            r->error = why;
        }
        L.queue.clear();
    }
    s.cv_done.notify_all();
    s.cv_work.notify_all();
}

void serve_loop(qlb_server* sp, int lane) {
    qlb_server& s = *sp;
    Lane& L = s.lanes[lane];
    Lane& other = s.lanes[lane ^ 1];
    cudaSetDevice(s.device);
    char* base = static_cast<char*>(s.arena_mem.p);
    std::unique_lock<std::mutex> lk(s.mu);
    while (true) {
        if (!s.fatal.empty()) break;
        admit(s, L);
        if (L.active.empty()) {
            if (s.stop && L.queue.empty()) break;
            s.cv_work.wait_for(lk, std::chrono::milliseconds(50));
            continue;
        }
        // While the other lane has work, the large lane leaves it a few SMs.
        const uint32_t cap = !other.active.empty() ? (lane == 1 ? static_cast<uint32_t>(sm_count()) - kSmallLaneCtas
                                                                : kSmallLaneCtas)
                                                   : 0u;
        // Requests admitted last round boundary need their program uploaded
        // and their state set to |0...0> before their first pass.
        std::vector<std::shared_ptr<Request>> batch = L.active;
        lk.unlock();
        cudaError_t e = cudaSuccess;
        auto* work = static_cast<TileWork*>(L.work_host.p);
        auto* meta = static_cast<char*>(L.meta_host.p);
        auto* bst = reinterpret_cast<BatchState*>(meta);
        auto* chunk_begin = reinterpret_cast<uint64_t*>(meta + align256(kMaxWork * sizeof(BatchState)));
        uint32_t nw = 0, nfin = 0;
        uint64_t tiles = 0, chunks = 0;
        int features = 0;
        std::vector<std::shared_ptr<Request>> finishing;
        for (auto& r : batch) {
            char* blk = base + r->block_off;
            if (r->next_pass == 0 && r->t_admit != 0 && e == cudaSuccess) {
                // first round of this request: program upload and |0...0>
                e = cudaMemcpyAsync(blk + r->o_pass, r->prog_image.data(), r->prog_image.size(),
                                    cudaMemcpyHostToDevice, L.stream);
                if (e == cudaSuccess)
                    e = cudaMemsetAsync(blk + r->o_state, 0, (size_t{1} << r->neff) * sizeof(float2), L.stream);
                if (e == cudaSuccess) {
                    const float2 one = make_float2(1.f, 0.f);
                    e = cudaMemcpyAsync(blk + r->o_state, &one, sizeof(float2), cudaMemcpyHostToDevice, L.stream);
                }
            }
            const uint32_t np = static_cast<uint32_t>(r->plan.steps.size());
            if (r->next_pass < np) {
                const PlanStep& st = r->plan.steps[r->next_pass];
                TileWork w{};
                w.state = reinterpret_cast<float2*>(blk + r->o_state);
                w.tile_begin = tiles;
                w.passes = reinterpret_cast<const TilePass*>(blk + r->o_pass);
                w.phases = reinterpret_cast<const TilePhase*>(blk + r->o_phase);
                w.ops = reinterpret_cast<const TileOp*>(blk + r->o_ops);
                w.mats = reinterpret_cast<const float2*>(blk + r->o_mat);
                w.pass = st.index;
                work[nw++] = w;
                tiles += uint64_t{1} << (r->neff - kTileQubits);
                features |= st.features;
            }
            if (r->next_pass + 1 >= np) {          // finishes this round
                bst[nfin] = BatchState{static_cast<uint64_t>((r->block_off + r->o_state) / sizeof(float2)), r->n,
                                       r->neff};
                chunk_begin[nfin] = chunks;
                chunks += uint64_t{1} << (r->neff - kBatchMinQubits);
                ++nfin;
                finishing.push_back(r);
            }
        }
        chunk_begin[nfin] = chunks;
        if (e == cudaSuccess && nw)
            e = cudaMemcpyAsync(L.work_dev.p, work, nw * sizeof(TileWork), cudaMemcpyHostToDevice, L.stream);
        if (e == cudaSuccess && nw)
            e = launch_tile_work(static_cast<const TileWork*>(L.work_dev.p), nw, tiles, features,
                                 static_cast<int*>(L.err_dev.p), L.stream, cap);
        if (e == cudaSuccess && nfin) {
            const size_t meta_bytes = align256(kMaxWork * sizeof(BatchState)) + (kMaxWork + 1) * sizeof(uint64_t);
            e = cudaMemcpyAsync(L.meta_dev.p, meta, meta_bytes, cudaMemcpyHostToDevice, L.stream);
            const auto* dst = static_cast<const BatchState*>(L.meta_dev.p);
            const auto* dcb = reinterpret_cast<const uint64_t*>(static_cast<const char*>(L.meta_dev.p) +
                                                                align256(kMaxWork * sizeof(BatchState)));
            if (e == cudaSuccess)
                e = launch_batch_expect_z(reinterpret_cast<const float2*>(base), dst, nfin, dcb, chunks,
                                          static_cast<double*>(L.partial_dev.p), static_cast<double*>(L.result_dev.p),
                                          kBatchStride, L.stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(L.result_host.p, L.result_dev.p, nfin * kBatchStride * sizeof(double),
                                    cudaMemcpyDeviceToHost, L.stream);
            for (auto& r : finishing) {
                if (e != cudaSuccess || r->shots == 0) continue;
                char* blk = base + r->block_off;
                e = launch_sample(reinterpret_cast<const float2*>(blk + r->o_state), r->neff, r->seed, r->shots,
                                  reinterpret_cast<double*>(blk + r->o_chunk),
                                  reinterpret_cast<uint64_t*>(blk + r->o_samples), L.stream);
            }
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(L.err_host.p, L.err_dev.p, sizeof(int), cudaMemcpyDeviceToHost, L.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(L.stream);
        // sample read-back (pageable destination: synchronous copies after the round)
        std::vector<std::vector<uint64_t>> smp(finishing.size());
        for (size_t i = 0; i < finishing.size() && e == cudaSuccess; ++i) {
            auto& r = finishing[i];
            smp[i].resize(r->shots);
            if (r->shots)
                e = cudaMemcpy(smp[i].data(), base + r->block_off + r->o_samples, r->shots * sizeof(uint64_t),
                               cudaMemcpyDeviceToHost);
        }
        const int dev_err = *static_cast<int*>(L.err_host.p);
        lk.lock();
        if (!s.fatal.empty()) break;   // the other lane failed while this round ran
        s.info.rounds += 1;
        s.info.launches += nw ? 1 : 0;
        s.info.tiles += tiles;
        if (e != cudaSuccess || dev_err) {
            // a CUDA failure or a bounded wait that gave up: fail everything in flight
            fail_all(s, e != cudaSuccess ? std::string("CUDA: ") + cudaGetErrorString(e)
                                         : std::string("a tile-kernel wait gave up"));
            break;
        }
        const double* res = static_cast<const double*>(L.result_host.p);
        for (size_t i = 0; i < finishing.size(); ++i) {
            auto& r = finishing[i];
            r->ez.assign(res + i * kBatchStride, res + i * kBatchStride + r->n);
            r->samples = std::move(smp[i]);
            r->status = REQ_DONE;
            r->t_done = s.now();
            s.arena.release(r->block_off, r->block_bytes);
            s.info.completed += 1;
        }
        for (auto& r : batch) r->next_pass += 1;
        // cancelled requests leave at the round boundary: their kernels are done
        bool dropped = false;
        for (auto& r : L.active)
            if (r->cancel && r->status == REQ_ACTIVE) {
                r->status = REQ_CANCELLED;
                r->t_done = s.now();
                s.arena.release(r->block_off, r->block_bytes);
                dropped = true;
            }
        L.active.erase(std::remove_if(L.active.begin(), L.active.end(),
                                      [](const std::shared_ptr<Request>& r) {
                                          return r->status == REQ_DONE || r->status == REQ_CANCELLED;
                                      }),
                       L.active.end());
        if (!finishing.empty() || dropped) {
            s.cv_done.notify_all();
            s.cv_work.notify_all();   // freed arena blocks: the other lane may admit
        }
    }
}

std::shared_ptr<Request> find(qlb_server& s, uint64_t id) {
    auto it = s.all.find(id);
    if (it == s.all.end()) fail(QLB_ERR_INVALID_ARG, "unknown request id");
    return it->second;
}

}  // namespace

extern "C" {

int qlb_server_create(qlb_server_t* out, const qlb_server_config* cfg) {
    return guarded([&] {
        need(out, "out");
        *out = nullptr;
        auto s = std::make_unique<qlb_server>();
        qlb_server_config c{};
        if (cfg) c = *cfg;
        if (c.mode != QLB_MODE_TILED && c.mode != QLB_MODE_TILED_TC) c.mode = QLB_MODE_TILED;
        s->mode = c.mode;
        s->fuse_from = c.fuse_from;
        s->max_active = c.max_active ? std::min<uint32_t>(c.max_active, kMaxWork) : kMaxWork;
        check_cuda(cudaGetDevice(&s->device), "device");
        size_t free_b = 0, total_b = 0;
        check_cuda(cudaMemGetInfo(&free_b, &total_b), "memory info");
        size_t bytes = c.memory_bytes ? c.memory_bytes : static_cast<size_t>(0.85 * static_cast<double>(free_b));
        bytes &= ~size_t{255};
        if (bytes < (size_t{1} << 20)) fail(QLB_ERR_OOM, "server arena below 1 MiB");
        s->arena_mem.ensure(bytes);
        s->arena.init(bytes);
        s->max_chunks = bytes / (sizeof(float2) << kBatchMinQubits) + 1;
        const size_t meta_bytes = align256(kMaxWork * sizeof(BatchState)) + (kMaxWork + 1) * sizeof(uint64_t);
        for (int i = 0; i < 2; ++i) {
            Lane& L = s->lanes[i];
            L.index = i;
            check_cuda(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking), "stream");
            L.partial_dev.ensure(batch_partial_doubles(s->max_chunks) * sizeof(double));
            L.result_dev.ensure(kMaxWork * kBatchStride * sizeof(double));
            L.result_host.ensure(kMaxWork * kBatchStride * sizeof(double));
            L.work_dev.ensure(kMaxWork * sizeof(TileWork));
            L.work_host.ensure(kMaxWork * sizeof(TileWork));
            L.meta_dev.ensure(meta_bytes);
            L.meta_host.ensure(meta_bytes);
            L.err_dev.ensure(256);
            L.err_host.ensure(sizeof(int));
            check_cuda(cudaMemsetAsync(L.err_dev.p, 0, sizeof(int), L.stream), "error flag");
            check_cuda(cudaStreamSynchronize(L.stream), "error flag");
        }
        check_cuda(configure_tile_kernel(), "tile kernel attributes");
        s->info.arena_bytes = bytes;
        for (int i = 0; i < 2; ++i) s->lanes[i].worker = std::thread(serve_loop, s.get(), i);
        *out = s.release();
    });
}

int qlb_server_submit(qlb_server_t s, const qlb_gate_instr* program, uint64_t count, const qlb_pool_view* pool,
                      uint32_t num_qubits, uint64_t shots, uint64_t seed, uint64_t* out_id) {
    return guarded([&] {
        need(s, "server");
        need(out_id, "out_id");
        if (count && !program) fail(QLB_ERR_INVALID_ARG, "program is null");
        if (num_qubits == 0 || num_qubits > 30) fail(QLB_ERR_INVALID_ARG, "served circuits take 1..30 qubits");
        static const qlb_pool_view empty{nullptr, 0, nullptr, 0};
        auto r = std::make_shared<Request>();
        r->n = num_qubits;
        r->neff = std::max(num_qubits, kBatchMinQubits);
        r->shots = shots;
        r->seed = seed;
        if (s->fuse_from && num_qubits >= s->fuse_from) {
            // the GPU middle end first: blocks of up to 5 qubits, no windowing
            // (the plan then holds them as tensor-core ops)
            qlb_transpile_config tc;
            qlb_transpile_config_default(&tc);
            tc.enable_hw_awareness = 0;
            tc.max_fusion_qubits = 5;
            qlb_module_t mod = nullptr;
            if (qlb_transpile_gpu(program, count, pool ? pool : &empty, num_qubits, &tc, &mod) != QLB_OK)
                fail(QLB_ERR_INVALID_ARG, std::string("request fusion: ") + qlb_last_error());
            struct Guard {
                qlb_module_t m;
                ~Guard() { qlb_module_destroy(m); }
            } guard{mod};
            const qlb_gate_instr* fp = nullptr;
            uint64_t fc = 0;
            qlb_pool_view fpool{};
            qlb_module_program(mod, &fp, &fc);
            qlb_module_pool(mod, &fpool);
            r->plan = plan_host(PlanConfig{r->neff, QLB_MODE_TILED_TC, 0, 10.0, 0}, fp, fc, &fpool);
        } else {
            r->plan = plan_host(PlanConfig{r->neff, s->mode, 0, 10.0, 0}, program, count, pool ? pool : &empty);
        }
        for (const PlanStep& st : r->plan.steps)
            if (st.kind != STEP_PASS)
                fail(QLB_ERR_INVALID_ARG, "served circuits may hold only gates (no MEASURE, no 6-qubit blocks)");
        const TileProgram& tp = r->plan.prog;
        // one arena block: state | passes | phases | ops | mats | chunk sums | samples
        size_t o = 0;
        r->o_state = o;
        o = align256(o + (size_t{1} << r->neff) * sizeof(float2));
        r->o_pass = o;
        const size_t rp = 0;
        const size_t rph = align256(rp + tp.passes.size() * sizeof(TilePass));
        const size_t rop = align256(rph + tp.phases.size() * sizeof(TilePhase));
        const size_t rmt = align256(rop + tp.ops.size() * sizeof(TileOp));
        const size_t rend = align256(rmt + tp.mats.size() * sizeof(float2));
        r->prog_image.assign(rend, 0);
        std::memcpy(r->prog_image.data() + rp, tp.passes.data(), tp.passes.size() * sizeof(TilePass));
        std::memcpy(r->prog_image.data() + rph, tp.phases.data(), tp.phases.size() * sizeof(TilePhase));
        std::memcpy(r->prog_image.data() + rop, tp.ops.data(), tp.ops.size() * sizeof(TileOp));
        std::memcpy(r->prog_image.data() + rmt, tp.mats.data(), tp.mats.size() * sizeof(float2));
        r->o_phase = r->o_pass + rph;
        r->o_ops = r->o_pass + rop;
        r->o_mat = r->o_pass + rmt;
        o = r->o_pass + rend;
        r->o_chunk = o;
        o = align256(o + sample_scratch_doubles(r->neff) * sizeof(double));
        r->o_samples = o;
        o = align256(o + shots * sizeof(uint64_t));
        r->block_bytes = o;
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->fatal.empty()) fail(QLB_ERR_CUDA, "server stopped: " + s->fatal);
        if (s->stop) fail(QLB_ERR_STATE, "server is shutting down");
        if (r->block_bytes > s->arena.capacity())
            fail(QLB_ERR_OOM, "request needs more device memory than the server arena holds");
        r->id = s->next_id++;
        r->t_submit = s->now();
        s->all[r->id] = r;
        s->lanes[r->n >= kLargeQubits ? 1 : 0].queue.push_back(r);
        s->info.submitted += 1;
        *out_id = r->id;
        s->cv_work.notify_all();
    });
}

int qlb_server_wait(qlb_server_t s, uint64_t id, double timeout_s) {
    return guarded([&] {
        need(s, "server");
        std::unique_lock<std::mutex> lk(s->mu);
        auto r = find(*s, id);
        const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
        auto settled = [&] {
            return r->status == REQ_DONE || r->status == REQ_FAILED || r->status == REQ_CANCELLED;
        };
        while (!settled()) {
            if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && !settled())
                fail(QLB_ERR_TIMEOUT, "request not finished within the timeout");
        }
        if (r->status == REQ_FAILED) fail(QLB_ERR_CUDA, r->error);
        if (r->status == REQ_CANCELLED) fail(QLB_ERR_STATE, "request was cancelled");
    });
}

int qlb_server_cancel(qlb_server_t s, uint64_t id) {
    return guarded([&] {
        need(s, "server");
        std::lock_guard<std::mutex> lk(s->mu);
        auto r = find(*s, id);
        if (r->status == REQ_QUEUED) {
            for (Lane& L : s->lanes)
                L.queue.erase(std::remove(L.queue.begin(), L.queue.end(), r), L.queue.end());
            r->status = REQ_CANCELLED;
            r->t_done = s->now();
            s->cv_done.notify_all();
        } else if (r->status == REQ_ACTIVE) {
            r->cancel = true;   // leaves at the next round boundary
        }
    });
}

int qlb_server_result(qlb_server_t s, uint64_t id, double* expect_z, uint32_t num_qubits, uint64_t* samples,
                      uint64_t shots, qlb_request_info* info) {
    return guarded([&] {
        need(s, "server");
        std::lock_guard<std::mutex> lk(s->mu);
        auto r = find(*s, id);
        if (r->status == REQ_FAILED) fail(QLB_ERR_CUDA, r->error);
        if (r->status == REQ_CANCELLED) {
            s->all.erase(id);
            fail(QLB_ERR_STATE, "request was cancelled");
        }
        if (r->status != REQ_DONE) fail(QLB_ERR_STATE, "request not finished");
        if (expect_z) {
            if (num_qubits != r->n) fail(QLB_ERR_INVALID_ARG, "expect_z length must equal the request's qubits");
            std::memcpy(expect_z, r->ez.data(), r->n * sizeof(double));
        }
        if (samples) {
            if (shots != r->shots) fail(QLB_ERR_INVALID_ARG, "samples length must equal the request's shots");
            std::memcpy(samples, r->samples.data(), r->shots * sizeof(uint64_t));
        }
        if (info) {
            info->num_qubits = r->n;
            info->passes = static_cast<uint32_t>(r->plan.steps.size());
            info->shots = r->shots;
            info->t_submit = r->t_submit;
            info->t_admit = r->t_admit;
            info->t_done = r->t_done;
        }
        s->all.erase(id);
    });
}

int qlb_server_stats(qlb_server_t s, qlb_server_info* out) {
    return guarded([&] {
        need(s, "server");
        need(out, "out");
        std::lock_guard<std::mutex> lk(s->mu);
        *out = s->info;
        out->queued = static_cast<uint32_t>(s->lanes[0].queue.size() + s->lanes[1].queue.size());
        out->active = static_cast<uint32_t>(s->lanes[0].active.size() + s->lanes[1].active.size());
        out->arena_used = s->arena.used();
    });
}

int qlb_server_destroy(qlb_server_t s) {
    return guarded([&] {
        if (!s) return;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
        }
        s->cv_work.notify_all();
        for (Lane& L : s->lanes)
            if (L.worker.joinable()) L.worker.join();
        delete s;
    });
}

}  // extern "C"

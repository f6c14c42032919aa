/*
 * qlassical_b200.h -- C ABI of the B200 execution backend for Qlassical.
 *
 * This is the drop-in boundary: the reference simulator's hot path is
 * CPUOpenMPEngine::execute over a transpiled IRModule
 * (include/backend/cpu_openmp_engine.hpp:143-225).  Every entry point below
 * replaces one member of the reference's ExecutionEngine / StateVector /
 * Middleware interfaces (cited per function) and takes only plain pointers,
 * sizes and opaque handles, so a C++20 wrapper (include/qlassical_b200/
 * cuda_engine.hpp), a ctypes binding or any other FFI can sit on top of it.
 *
 * Conventions (identical to the reference):
 *   - qubit q <-> bit q of the amplitude index (little endian);
 *   - dense matrices are row-major, matrix-index bit i <-> instr.qubits[i]
 *     (cpu_openmp_engine.hpp:558-566);
 *   - host amplitudes are interleaved complex128 (std::complex<double>),
 *     device amplitudes are complex64 (float2), 256-byte aligned.
 *
 * Every function returns a qlb_status.  No C++ exception crosses the ABI;
 * qlb_last_error() returns a thread-local message for the last failure.
 */
#ifndef QLASSICAL_B200_H
#define QLASSICAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Wire format                                                              */
/* ------------------------------------------------------------------------ */

/* Gate type codes: the values of qlassical::GateType (frontend.hpp:26-51),
 * plus two additive diagonal types (CZ, CP) in the free two-qubit range. */
enum qlb_gate_type {
    QLB_H = 0x00, QLB_X = 0x01, QLB_Y = 0x02, QLB_Z = 0x03, QLB_S = 0x04,
    QLB_RX = 0x10, QLB_RY = 0x11, QLB_RZ = 0x12,
    QLB_CX = 0x20, QLB_SWAP = 0x21,
    QLB_CZ = 0x22,          /* additive: diag(1,1,1,-1) on (qubits[0], qubits[1]) */
    QLB_CP = 0x23,          /* additive: diag(1,1,1,e^{i*param}) */
    QLB_CCX = 0x30, QLB_CSWAP = 0x31,
    QLB_UNITARY = 0x80,
    QLB_FUSED_BLOCK = 0xE0, QLB_GLOBAL_SWAP = 0xE1,
    QLB_BARRIER = 0xF0, QLB_MEASURE = 0xF1
};

/* Byte-for-byte the layout of qlassical::GateInstr (frontend.hpp:84-105):
 * offsets 0/1/2/8/12, 16 bytes, 16-byte aligned.  The reference's two pad
 * bytes (offset 6-7) carry qubits 4 and 5 of a 5- or 6-qubit FUSED_BLOCK or
 * UNITARY; they stay 0 for every other instruction, which the reference
 * ignores, so streams remain readable by the reference engine. */
typedef struct qlb_gate_instr {
    uint8_t type;
    uint8_t flags_arity;       /* low nibble: arity, high nibble: flags */
    uint8_t qubits[4];
    uint8_t qubits_ext[2];     /* reference: uint16_t _pad */
    union { float param; uint32_t matrix_idx; } payload;
    uint32_t uid;
} qlb_gate_instr;

/* UnitaryPool::MatrixEntry (frontend.hpp:118-123): 12 bytes. */
typedef struct qlb_matrix_entry {
    uint32_t offset;           /* start index (in complex elements) into data */
    uint32_t num_elements;     /* 4^k */
    uint8_t  num_qubits;       /* k */
    uint8_t  pad[3];
} qlb_matrix_entry;

/* A read-only view of a UnitaryPool (frontend.hpp:117-164):
 * data = interleaved complex128, 2*num_elements doubles. */
typedef struct qlb_pool_view {
    const double*           data;
    uint64_t                num_elements;
    const qlb_matrix_entry* metadata;
    uint64_t                num_matrices;
} qlb_pool_view;

/* ------------------------------------------------------------------------ */
/* Status                                                                   */
/* ------------------------------------------------------------------------ */

typedef enum qlb_status {
    QLB_OK = 0,
    QLB_ERR_INVALID_ARG = 1,   /* -> std::invalid_argument */
    QLB_ERR_OOM = 2,           /* -> std::bad_alloc */
    QLB_ERR_CUDA = 3,          /* -> std::runtime_error */
    QLB_ERR_UNKNOWN_GATE = 4,  /* -> std::runtime_error (cpu_openmp_engine.hpp:221-222) */
    QLB_ERR_NOT_NORMALIZED = 5,/* -> std::invalid_argument (cpu_state_vector.hpp:97-106) */
    QLB_ERR_TIMEOUT = 6,       /* a bounded device wait gave up */
    QLB_ERR_STATE = 7          /* call order violated (e.g. empty state) */
} qlb_status;

const char* qlb_last_error(void);
/* Library version string and the CUDA device it will use. */
const char* qlb_version(void);
/* Selects the CUDA device used by later calls from this thread (the library
 * links its own CUDA runtime, so a host framework's current device is not
 * inherited). */
int qlb_set_device(int device);
int qlb_device_info(int* sm_count, uint64_t* free_bytes, uint64_t* total_bytes);
/* Failure-path self-test (no reference counterpart): runs the device wait
 * that the tile kernel uses for copy and tensor-core completions on a
 * barrier that nothing completes, with a limit of limit_ms (1..2000).  The
 * wait must give up and report: *gave_up = 1, and the CUDA context stays
 * usable.  Every wait of the tile kernel is bounded this way (2 s); when one
 * gives up, the call that launched it returns QLB_ERR_TIMEOUT. */
int qlb_selftest_bounded_wait(uint32_t limit_ms, int* gave_up);

/* ------------------------------------------------------------------------ */
/* CUDAStateVector (replaces CPUStateVector, cpu_state_vector.hpp:24-162)   */
/* ------------------------------------------------------------------------ */

typedef struct qlb_state* qlb_state_t;

int qlb_state_create(qlb_state_t* out);                                  /* CPUStateVector() */
int qlb_state_destroy(qlb_state_t sv);
int qlb_state_initialize(qlb_state_t sv, uint32_t num_qubits);           /* :54-78  */
int qlb_state_initialize_from(qlb_state_t sv, const double* amps_c128,
                              uint64_t dim);                             /* :82-115 */
int qlb_state_num_qubits(qlb_state_t sv, uint32_t* out);                 /* :148-150 */
int qlb_state_dimension(qlb_state_t sv, uint64_t* out);                  /* :152-154 */
int qlb_state_empty(qlb_state_t sv, int* out);                           /* :156-158 */
int qlb_state_download(qlb_state_t sv, double* out_c128, uint64_t dim);  /* amplitudes() */
int qlb_state_device_ptr(qlb_state_t sv, void** out_float2);             /* data() */

/* ------------------------------------------------------------------------ */
/* CUDAEngine (replaces CPUOpenMPEngine, cpu_openmp_engine.hpp:51-672)      */
/* ------------------------------------------------------------------------ */

typedef struct qlb_engine* qlb_engine_t;

/* Execution strategies for execute():
 *  PLAIN    - one HBM sweep per instruction (the plain GPU path);
 *  TILED    - runs of instructions applied inside shared-memory tiles,
 *             dense blocks on FP32 CUDA cores;
 *  TILED_TC - as TILED, dense blocks of >= 4 qubits on the tensor cores
 *             (tcgen05, split-precision bf16, FP32 accumulate). */
enum qlb_exec_mode { QLB_MODE_PLAIN = 0, QLB_MODE_TILED = 1, QLB_MODE_TILED_TC = 2 };

int qlb_engine_create(qlb_engine_t* out, uint32_t num_qubits, int has_seed,
                      uint64_t seed, uint64_t reserve_meas);             /* :65-80   */
int qlb_engine_create_from_amplitudes(qlb_engine_t* out, const double* amps_c128,
                      uint64_t dim, int has_seed, uint64_t seed,
                      uint64_t reserve_meas);                            /* :87-102  */
int qlb_engine_create_from_state(qlb_engine_t* out, qlb_state_t sv);     /* :105-107 (moves sv) */
int qlb_engine_destroy(qlb_engine_t e);
int qlb_engine_set_state_vector(qlb_engine_t e, qlb_state_t sv);         /* :110-112 (moves sv) */
int qlb_engine_extract_state_vector(qlb_engine_t e, qlb_state_t out_sv); /* :245-247 (moves into out_sv) */
int qlb_engine_reset(qlb_engine_t e);                                    /* :119-122 */
int qlb_engine_reset_to(qlb_engine_t e, const double* amps_c128, uint64_t dim); /* :125-128 */
int qlb_engine_set_seed(qlb_engine_t e, uint64_t seed);                  /* :130-132 */
int qlb_engine_reserve_measurements(qlb_engine_t e, uint64_t count);     /* :134-136 */
int qlb_engine_measurements(qlb_engine_t e, const uint8_t** data, uint64_t* count); /* :138-140 */
int qlb_engine_execute(qlb_engine_t e, const qlb_gate_instr* program,
                       uint64_t count, const qlb_pool_view* pool);       /* :143-225 */
int qlb_engine_state(qlb_engine_t e, double* out_c128, uint64_t dim);    /* :231-233 (D2H + widen) */
int qlb_engine_num_qubits(qlb_engine_t e, uint32_t* out);                /* :235-237 */
int qlb_engine_set_mode(qlb_engine_t e, int mode);
int qlb_engine_get_mode(qlb_engine_t e, int* mode);
/* Engine options.  QLB_OPT_PHYSICAL_GLOBAL_SWAP = 1 makes GLOBAL_SWAP move
 * data (one bandwidth-bound swap pass each, logical order restored when
 * execute() returns); 0 (default) applies the permutation lazily by
 * re-addressing later instructions, which gives the same state with no
 * data movement.  QLB_OPT_TC_MIN_COST (TILED_TC only): a run of
 * register-local ops goes to the tensor cores when its estimated CUDA-core
 * cost, in hundredths of an instruction per amplitude, reaches the value
 * (default 1000); cheaper runs stay on the CUDA cores.  QLB_OPT_TC_CHAIN
 * (TILED_TC only, default 1): a register phase whose ops are all uniform
 * over the tile becomes one tensor-core op whatever its cost, and a pass
 * made only of such phases runs on the tensor-core chain kernel (two tiles
 * in flight per SM, loads by a dedicated warp); 0 keeps every pass on the
 * general tile kernel.  QLB_OPT_TILE_LOW (tiled modes, 3..6, default 3):
 * memory qubits 0..value-1 belong to every tile, so a tile is read and
 * written in contiguous runs of 2^value amplitudes; the other 13 - value
 * tile qubits are chosen per pass.  The batched autotuner searches it. */
enum qlb_option { QLB_OPT_PHYSICAL_GLOBAL_SWAP = 1, QLB_OPT_TC_MIN_COST = 2, QLB_OPT_TC_CHAIN = 3,
                  QLB_OPT_TILE_LOW = 4 };
int qlb_engine_set_option(qlb_engine_t e, int key, int64_t value);
int qlb_engine_synchronize(qlb_engine_t e);
/* The device state pointer (float2 *) and the stream the engine launches on. */
int qlb_engine_device_state(qlb_engine_t e, void** out_float2);
int qlb_engine_stream(qlb_engine_t e, void** out_cuda_stream);
/* Statistics of the last execute(): HBM sweeps, kernel launches, tile passes. */
typedef struct qlb_exec_stats {
    uint64_t instructions;      /* instructions in the program */
    uint64_t sweeps;            /* full-state HBM read+write passes executed */
    uint64_t launches;          /* kernels launched */
    uint64_t tile_passes;       /* tiled passes (subset of sweeps) */
    uint64_t permute_passes;    /* qubit-permutation passes (subset of sweeps) */
    uint64_t dense_ops;         /* dense unitaries applied */
    uint64_t tc_ops;            /* dense unitaries applied on the tensor cores */
    double   sweep_bytes;       /* algorithmic bytes: 16 B/amp per full sweep */
    uint64_t chain_passes;      /* tiled passes run by the tensor-core chain kernel */
} qlb_exec_stats;
int qlb_engine_last_stats(qlb_engine_t e, qlb_exec_stats* out);

/* Compiled programs.  execute() == compile + run + destroy.  A plan holds the
 * engine-ready form of one program (its pass schedule and every operand
 * already in device memory) for one qubit count and execution mode, so it
 * can be run many times with no host work besides the launches.  Running a
 * plan whose qubit count differs from the engine's state is an error. */
typedef struct qlb_plan* qlb_plan_t;
int qlb_engine_compile(qlb_engine_t e, const qlb_gate_instr* program, uint64_t count,
                       const qlb_pool_view* pool, qlb_plan_t* out);
int qlb_engine_run(qlb_engine_t e, qlb_plan_t plan);
int qlb_plan_stats(qlb_plan_t plan, qlb_exec_stats* out);
int qlb_plan_destroy(qlb_plan_t plan);
/* EXPLAIN: runs the planner on the host only (no GPU needed) for a state of
 * num_qubits and returns the plan as JSON -- steps, passes (tile qubits,
 * register phases), per-phase ops and their matrices.  Writes at most `cap`
 * bytes (NUL-terminated) and the full length to *needed. */
int qlb_describe_plan(uint32_t num_qubits, int mode, int physical_global_swap,
                      const qlb_gate_instr* program, uint64_t count, const qlb_pool_view* pool,
                      char* out, uint64_t cap, uint64_t* needed);
/* The same with the planner options an engine takes from QLB_OPT_TILE_LOW
 * (tile_low, 3..6) and QLB_OPT_TC_CHAIN (tc_chain); qlb_describe_plan is
 * tile_low 3, tc_chain 1. */
int qlb_describe_plan_opts(uint32_t num_qubits, int mode, int physical_global_swap, int tile_low, int tc_chain,
                           const qlb_gate_instr* program, uint64_t count, const qlb_pool_view* pool,
                           char* out, uint64_t cap, uint64_t* needed);

/* FP64 reductions over the device state (no reference counterpart except
 * the probability reduction inside apply_measure, :622-630). */
int qlb_engine_norm_sq(qlb_engine_t e, double* out);
int qlb_engine_prob_one(qlb_engine_t e, uint32_t qubit, double* out);
int qlb_engine_expect_z(qlb_engine_t e, double* out, uint32_t num_qubits);
/* FP64 checker (no counterpart in the reference engine, whose arithmetic is
 * complex128 on the host, cpu_openmp_engine.hpp:143-225): a complex128
 * state on the device that runs a program gate by gate in double precision,
 * for measuring the complex64 engine's error at sizes a host complex128 run
 * cannot reach in reasonable time (30 qubits: 17.2 GB).  It accepts every
 * instruction type except MEASURE; GLOBAL_SWAP permutes physical qubits and
 * the state stays in logical order, as the engine's does.
 * qlb_check64_compare() reduces, over the whole state and in FP64, the
 * difference between the checker's state and a complex64 device state of
 * the same size (e.g. qlb_engine_device_state()). */
typedef struct qlb_check64* qlb_check64_t;
typedef struct qlb_check64_result {
    double max_abs_diff;   /* max_i |ref_i - psi_i| */
    double infidelity;     /* 1 - |<ref|psi>|^2 / (<ref|ref> <psi|psi>) */
    double norm_ref, norm_state;
    double overlap_re, overlap_im;   /* <ref|psi> */
} qlb_check64_result;
int qlb_check64_create(qlb_check64_t* out, uint32_t num_qubits);          /* |0...0>, 1..33 qubits */
int qlb_check64_execute(qlb_check64_t c, const qlb_gate_instr* program, uint64_t count,
                        const qlb_pool_view* pool);
int qlb_check64_compare(qlb_check64_t c, const void* state_float2, qlb_check64_result* out);
int qlb_check64_download(qlb_check64_t c, double* out_c128, uint64_t dim);
int qlb_check64_destroy(qlb_check64_t c);

/* <Z_q> for every qubit of a complex64 device state, allocating nothing.
 * No counterpart in the reference.  For callers that must not allocate
 * device memory while they run -- such as a serving loop that admits
 * requests by accounting all free HBM to resident state vectors, where a
 * hidden cudaMalloc would escape that accounting and cudaMalloc/cudaFree
 * would synchronize the device under other requests' kernels.  The
 * reduction's scratch is a fixed ~176 KiB array inside the library that
 * every GPU loading the library holds until exit.  Accepts 1..34 qubits
 * (rejects others with QLB_ERR_INVALID_ARG).  `out` is host memory for
 * num_qubits doubles; the call runs on `cuda_stream` and waits for it.
 * All calls share the scratch: calls whose kernels overlap on the GPU race,
 * so serialize them.  The first call on a device looks up the scratch's
 * device address with that device current, which is also when the device
 * commits the scratch (the library's modules load lazily): make that first
 * call -- a warm-up on any small state -- before any stream capture starts
 * and before measuring the free memory to be budgeted. */
int qlb_expect_z_noalloc(const void* state_float2, uint32_t num_qubits, double* out, void* cuda_stream);
/* Draws `shots` basis states from |amp|^2 with a counter-based generator
 * keyed by `seed`; identical seeds give identical samples on any launch. */
int qlb_engine_sample(qlb_engine_t e, uint64_t seed, uint64_t shots, uint64_t* out);
/* Amplitudes at chosen indices (complex128, `count` of them): a device-side
 * gather, for states too large to download (the reference's state() view
 * has no GPU equivalent at 33 qubits). */
int qlb_engine_amplitudes_at(qlb_engine_t e, const uint64_t* indices, uint64_t count, double* out_c128);

/* ------------------------------------------------------------------------ */
/* GPU middle end (replaces Middleware::transpile_gpu, middleware.hpp:866)  */
/* ------------------------------------------------------------------------ */

/* WindowingCostModel::evaluate_swap (middleware.hpp:50-53) as a C callback:
 * return 1 and fill (*active, *victim) -- logical qubits -- to request a
 * swap, 0 for none. */
typedef int (*qlb_cost_model_fn)(void* ctx, const uint32_t* window_frequencies,
                                 const uint16_t* log_to_phys, const uint16_t* phys_to_log,
                                 uint32_t num_qubits, uint16_t* active, uint16_t* victim);

typedef struct qlb_transpile_config {
    int      enable_gate_fusion;   /* TranspilerConfig::enable_gate_fusion (:363) */
    int      enable_hw_awareness;  /* TranspilerConfig::enable_hw_awareness (:364) */
    int      cost_model_type;      /* 0 THRESHOLD, 1 GREEDY, 2 CUSTOM (:352-356) */
    uint32_t numa_penalty;         /* (:370) */
    uint32_t swap_penalty;         /* (:371) */
    int      k_safe;               /* <0: from the GPU topology (the tile window) */
    int      max_fusion_qubits;    /* 1..6; the reference's limit is 4 (:137) */
    int      reference_fusable_set;/* 1: only H,X,Y,Z,S,CX,UNITARY,FUSED_BLOCK fuse (:442-448) */
    qlb_cost_model_fn custom_cost_model;   /* TranspilerConfig::custom_cost_model (:379) */
    void*    custom_cost_model_ctx;
} qlb_transpile_config;

typedef struct qlb_module* qlb_module_t;

void qlb_transpile_config_default(qlb_transpile_config* cfg);
int qlb_transpile_gpu(const qlb_gate_instr* program, uint64_t count,
                      const qlb_pool_view* pool, uint32_t num_qubits,
                      const qlb_transpile_config* cfg, qlb_module_t* out);
int qlb_module_destroy(qlb_module_t m);
int qlb_module_program(qlb_module_t m, const qlb_gate_instr** program, uint64_t* count);
int qlb_module_pool(qlb_module_t m, qlb_pool_view* out);
/* GPUTopology::get_safe_qubit_limit(): the shared-memory tile window. */
int qlb_gpu_safe_qubit_limit(uint32_t* out);

/* ------------------------------------------------------------------------ */
/* Batched mode: many independent circuits per launch.  No counterpart in   */
/* the reference (its engine runs one circuit per CPUOpenMPEngine); the     */
/* per-circuit semantics are execute() on |0...0> followed by <Z_i>.        */
/* ------------------------------------------------------------------------ */

typedef struct qlb_batch* qlb_batch_t;

/* The batched autotuner (mode -1) times QLB_BATCH_TUNE_CANDIDATES planner
 * configurations per size class -- the circuits of one padded qubit count,
 * 13..30: candidate i runs mode QLB_MODE_TILED (i < 3) or QLB_MODE_TILED_TC
 * (i >= 3) with 3 + i % 3 fixed low tile qubits (QLB_OPT_TILE_LOW), each on
 * a sample of the class (its first circuits, about two tiles per SM, at most
 * 128) by CUDA events around three runs of the sample's tile rounds.  A
 * round launches one kernel body for all its passes, so the mode is chosen
 * for the whole batch (the smaller total of the classes' best candidates in
 * that mode, projected to the class sizes) and the fixed low qubits per
 * class. */
#define QLB_BATCH_TUNE_CANDIDATES 6
#define QLB_BATCH_TUNE_CLASSES 18
typedef struct qlb_batch_tune_class {
    uint32_t num_qubits;    /* padded qubit count (13..30) */
    uint32_t circuits;      /* circuits of the class in the batch */
    uint32_t sample;        /* circuits timed per candidate */
    int32_t  best;          /* the candidate that plans the class (in the batch's mode) */
    float    ms[QLB_BATCH_TUNE_CANDIDATES];  /* sample time per candidate; < 0: the candidate failed to plan */
} qlb_batch_tune_class;

typedef struct qlb_batch_info {
    uint32_t circuits;
    uint32_t rounds;        /* tile-kernel launches = max passes over the circuits */
    int      mode;          /* QLB_MODE_TILED or QLB_MODE_TILED_TC; -1: size classes differ */
    uint32_t launches;      /* kernel launches per run */
    uint64_t tiles;         /* 2^13-amplitude tiles processed per run */
    uint64_t passes;        /* sum over circuits of executed passes */
    uint64_t amp_updates;   /* sum over circuits of (gates * 2^num_qubits) */
    uint64_t state_bytes;   /* device bytes of all state vectors */
    double   autotune_ms[2];/* mode -1: the tile rounds of the whole batch projected from the
                               samples: [0] the chosen configuration, [1] candidate 0 everywhere */
    double   tune_seconds;  /* mode -1: host time of the search (sample planning and timing) */
    uint32_t tune_classes;  /* mode -1: entries of tune[] in use */
    uint32_t pad;
    qlb_batch_tune_class tune[QLB_BATCH_TUNE_CLASSES];
    double   fuse_seconds;  /* host time of the circuits' fusion (qlb_batch_create_ex) */
    double   plan_seconds;  /* host time of the final planning, assembly and graph capture */
} qlb_batch_info;

/* Plans `count` circuits (program c: counts[c] instructions over pools[c],
 * num_qubits[c] in 1..30; gates only -- no MEASURE or 6-qubit blocks),
 * allocates every state vector and captures one CUDA graph per run.
 * mode: QLB_MODE_TILED, QLB_MODE_TILED_TC (3 fixed low tile qubits), or -1
 * to autotune each size class (above). */
int qlb_batch_create(qlb_batch_t* out, uint32_t count, const qlb_gate_instr* const* programs,
                     const uint64_t* counts, const qlb_pool_view* pools, const uint32_t* num_qubits,
                     int mode);
/* The same, with every circuit first fused by the GPU middle end
 * (qlb_transpile_gpu: blocks of up to fuse_qubits <= 5 qubits, no windowing)
 * on host threads; 0 = no fusion (qlb_batch_create).  Fused blocks run best
 * on the tensor cores (QLB_MODE_TILED_TC, or -1 to autotune). */
int qlb_batch_create_ex(qlb_batch_t* out, uint32_t count, const qlb_gate_instr* const* programs,
                        const uint64_t* counts, const qlb_pool_view* pools, const uint32_t* num_qubits,
                        int mode, uint32_t fuse_qubits);
/* Resets every state to |0...0>, runs all circuits and the FP64 <Z_i>
 * reductions: one graph launch on the batch's stream (asynchronous). */
int qlb_batch_run(qlb_batch_t b);
/* Waits for the run; QLB_ERR_TIMEOUT if a bounded device wait gave up. */
int qlb_batch_synchronize(qlb_batch_t b);
/* <Z_q> of circuit c into out[c * stride + q], q < num_qubits[c]. */
int qlb_batch_expect_z(qlb_batch_t b, double* out, uint32_t stride);
/* Amplitudes of circuit `index` (complex128, dim = 2^num_qubits). */
int qlb_batch_state(qlb_batch_t b, uint32_t index, double* out_c128, uint64_t dim);
int qlb_batch_stats(qlb_batch_t b, qlb_batch_info* out);
int qlb_batch_stream(qlb_batch_t b, void** out_cuda_stream);
int qlb_batch_destroy(qlb_batch_t b);

/* ------------------------------------------------------------------------ */
/* Serving loop: continuous batching of independent requests on one GPU.   */
/* No counterpart in the reference.  A request = (circuit, shots, seed)    */
/* run from |0...0>; its result = <Z_i> (FP64) and `shots` basis-state     */
/* samples (counter-based, keyed by (seed, shot)).  Requests are admitted  */
/* in arrival order while their state vector, program and sampling scratch */
/* fit in a device arena reserved at creation, and join the running rounds */
/* at the next round boundary (one tile pass per request per round).  A    */
/* request's results do not depend on which requests share its rounds.    */
/* ------------------------------------------------------------------------ */

typedef struct qlb_server* qlb_server_t;

typedef struct qlb_server_config {
    uint64_t memory_bytes;  /* device arena; 0 = 85% of the free HBM at creation */
    int      mode;          /* QLB_MODE_TILED (default) or QLB_MODE_TILED_TC */
    uint32_t max_active;    /* admitted requests at once; 0 = 4096 */
    uint32_t fuse_from;     /* requests of at least this many qubits are first fused by the GPU
                               middle end (qlb_transpile_gpu: blocks of up to 5 qubits, no
                               windowing) and planned for the tensor cores; 0 = never */
    uint32_t pad;
} qlb_server_config;

typedef struct qlb_server_info {
    uint64_t submitted, completed, rounds, launches, tiles;
    uint32_t queued, active;
    uint64_t arena_bytes, arena_used;
} qlb_server_info;

typedef struct qlb_request_info {
    uint32_t num_qubits, passes;
    uint64_t shots;
    double   t_submit, t_admit, t_done;   /* seconds since the server started */
} qlb_request_info;

int qlb_server_create(qlb_server_t* out, const qlb_server_config* cfg);
/* Plans the circuit on the calling thread and queues it (gates only, 1..30
 * qubits); QLB_ERR_OOM if it can never fit the arena. */
int qlb_server_submit(qlb_server_t s, const qlb_gate_instr* program, uint64_t count,
                      const qlb_pool_view* pool, uint32_t num_qubits, uint64_t shots,
                      uint64_t seed, uint64_t* out_request_id);
/* Blocks until the request finished (QLB_ERR_TIMEOUT after timeout_s;
 * QLB_ERR_STATE if it was cancelled). */
int qlb_server_wait(qlb_server_t s, uint64_t request_id, double timeout_s);
/* Cancels a request: a queued one leaves the queue at once, an admitted one
 * at the next round boundary (its device memory is then released).  No
 * effect on a finished request. */
int qlb_server_cancel(qlb_server_t s, uint64_t request_id);
/* Copies a finished request's results (either pointer may be NULL) and
 * forgets the request. */
int qlb_server_result(qlb_server_t s, uint64_t request_id, double* expect_z, uint32_t num_qubits,
                      uint64_t* samples, uint64_t shots, qlb_request_info* info);
int qlb_server_stats(qlb_server_t s, qlb_server_info* out);
/* Finishes every submitted request, then stops the server thread. */
int qlb_server_destroy(qlb_server_t s);

#ifdef __cplusplus
}
#endif

#endif /* QLASSICAL_B200_H */

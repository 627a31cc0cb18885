/*
 * dqsim_sv.h - C ABI of the B200 dense-statevector engine.
 *
 * This is the drop-in seam for dqsim's StatevectorSimulator backend.  The
 * reference binds the same operations through PyO3; every entry point below
 * names the reference method it replaces (paths relative to the dqsim project
 * root).  All functions return a dq_status; on failure dq_last_error() holds
 * a message for the calling thread.  No C++ exceptions cross this boundary,
 * no torch or CUDA types appear in the signatures, and every buffer is a
 * plain host pointer with an explicit size.
 *
 * Conventions (src/types.rs, docs/simulators.md:5-90):
 *   - circuits are the transport JSON produced by model_dump_json();
 *   - amplitudes are little-endian: qubit 0 is the least significant bit;
 *   - query qubit lists put their first qubit in the most significant bit;
 *   - count keys are '0'/'1' strings, classical bit 0 rightmost.
 */
#ifndef DQSIM_SV_H
#define DQSIM_SV_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DQ_API __attribute__((visibility("default")))
#else
#define DQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; each maps to the Python exception the reference raises. */
typedef enum dq_status {
    DQ_OK = 0,
    DQ_VALUE_ERROR = 1,     /* ValueError: parse, validation, query, options */
    DQ_MEMORY_ERROR = 2,    /* MemoryError: budget or allocation failure */
    DQ_TYPE_ERROR = 3,      /* TypeError: unsupported option */
    DQ_RUNTIME_ERROR = 4,   /* RuntimeError: profile write, nonfinite norm */
    DQ_NOT_IMPLEMENTED = 5, /* NotImplementedError: backend not provided */
    DQ_CUDA_ERROR = 6       /* RuntimeError: CUDA failure */
} dq_status;

typedef enum dq_precision {
    DQ_COMPLEX128 = 0, /* plain form: complex128 state, per-operation FP64 kernels */
    DQ_COMPLEX64 = 1   /* fused form: complex64 state, fused <=5-qubit blocks */
} dq_precision;

typedef struct dq_sim dq_sim;
typedef struct dq_result dq_result;
typedef struct dq_counts dq_counts;

/* Constructor options of StatevectorSimulator.__new__
 * (src/monolithic/statevector/simulator.rs:225-254). */
typedef struct dq_sim_options {
    int has_seed;
    uint64_t seed;
    int profile;
    uint64_t max_memory_mb;      /* default 1024; the budget of device working memory */
    int has_max_parallel_shots;
    uint64_t max_parallel_shots; /* concurrent device trajectories */
    int sample_terminal;         /* default 1 */
    int precision;               /* dq_precision, default DQ_COMPLEX128 */
    int device;                  /* CUDA device ordinal, default 0 */
    int execution;               /* 0 auto (shared-memory tile passes), 1 per-gate, 2 tiled */
    int tile_qubits;             /* qubits per shared-memory tile; 0 = 12 (complex128) / 13 (complex64) */
    int fusion_width;            /* widest fused dense operation inside a tile; 0 = 2 */
} dq_sim_options;

/* Per-category counters of SimulationProfile (simulator.rs:43-59). */
typedef struct dq_profile {
    uint64_t apply_one_qubit_calls;
    double apply_one_qubit_time;
    uint64_t apply_n_qubit_calls;
    double apply_n_qubit_time;
    uint64_t measure_qubit_calls;
    double measure_qubit_time;
    double total_time;
} dq_profile;

/* Message of the last failed call on this thread ("" if none). */
DQ_API const char* dq_last_error(void);

/* Library version string. */
DQ_API const char* dq_version(void);

/* Fill `opts` with the reference's defaults. */
DQ_API void dq_sim_options_default(dq_sim_options* opts);

/* StatevectorSimulator(seed, profile, *, max_memory_mb, max_parallel_shots,
 * sample_terminal): simulator.rs:225-254.  Checks options only; the CUDA
 * device is opened on first use. */
DQ_API int dq_sim_create(const dq_sim_options* opts, dq_sim** out);
DQ_API void dq_sim_destroy(dq_sim* sim);

/* StatevectorSimulator.simulate_shots(circuit, shots, profile):
 * simulator.rs:258-317 with run_shots, shots.rs:59-260.  With profile set,
 * writes dqsim_profiles/statevector_shots_profile_<ns>.json. */
DQ_API int dq_simulate_shots(dq_sim* sim, const char* json, size_t json_len, uint64_t shots, int profile,
                      dq_counts** out);

/* StatevectorSimulator.simulate(circuit): simulator.rs:320-371 (one trajectory). */
DQ_API int dq_simulate(dq_sim* sim, const char* json, size_t json_len, dq_result** out);

/* Count maps: `key_width` characters per key, keys concatenated without separators. */
DQ_API int dq_counts_size(const dq_counts* c, uint64_t* n_keys, uint64_t* key_width);
DQ_API int dq_counts_copy(const dq_counts* c, char* keys, uint64_t* counts);
DQ_API void dq_counts_free(dq_counts* c);

/* SimulationResult (simulator.rs:85-191). */
DQ_API int dq_result_num_qubits(const dq_result* r, uint64_t* n);
DQ_API int dq_result_num_cbits(const dq_result* r, uint64_t* n);
/* .statevector: 2 * 2^n doubles (re, im interleaved), an independent copy. */
DQ_API int dq_result_statevector(const dq_result* r, double* out, uint64_t out_len);
/* .classical_bits: one byte (0/1) per classical bit. */
DQ_API int dq_result_classical_bits(const dq_result* r, uint8_t* out, uint64_t out_len);
/* .profile: *has = 0 when the simulator ran without profiling. */
DQ_API int dq_result_profile(const dq_result* r, dq_profile* out, int* has);
/* .probabilities(qubits): out receives 2^k doubles; qubits[0] is the MSB.
 * has_qubits = 0 selects all qubits in descending order. */
DQ_API int dq_result_probabilities(const dq_result* r, const uint64_t* qubits, size_t k, int has_qubits, double* out,
                            uint64_t out_len);
/* .counts(shots, qubits, seed): keys are k-bit strings, qubits[0] leftmost.
 * has_seed = 0 draws a fresh seed. */
DQ_API int dq_result_counts(const dq_result* r, uint64_t shots, const uint64_t* qubits, size_t k, int has_qubits,
                     uint64_t seed, int has_seed, dq_counts** out);
/* .fidelity(other): |<self|other>|^2; 0.0 when the lengths differ. */
DQ_API int dq_result_fidelity(const dq_result* r, const double* other, uint64_t other_len, double* out);

/* Amplitudes of the result's state at `count` indices (little-endian basis
 * index, qubit 0 = LSB), written as 2*count doubles (re, im), read on the device
 * without copying the state to the host.  Extra query: the reference's
 * statevector result has no counterpart; it mirrors the MPS / P-block results'
 * `amplitude` (src/monolithic/mps/result.rs:114-130,
 * src/distributed/pblock/result.rs:141).  Out-of-range index -> DQ_VALUE_ERROR. */
DQ_API int dq_result_amplitudes(const dq_result* r, const uint64_t* indices, uint64_t count, double* out);

/* <psi|P|psi> for the Pauli product P with X on the bits of x_mask & ~z_mask,
 * Z on z_mask & ~x_mask and Y on x_mask & z_mask (qubit q = bit q), reduced in
 * FP64 on the device; *re is the expectation, *im its (rounding-level)
 * imaginary part.  Extra query mirroring the MPS result's `expectation_value`
 * (src/monolithic/mps/result.rs:209-236); no statevector counterpart. */
DQ_API int dq_result_pauli_expectation(const dq_result* r, uint64_t x_mask, uint64_t z_mask, double* re, double* im);
DQ_API void dq_result_free(dq_result* r);

/* Prepared circuits: parse, validate, compile and lower once, keep the state
 * and sampling buffers resident, then run repeatedly.  The reference reuses a
 * compiled plan and one prefix evolution for every shot of a call
 * (src/monolithic/statevector/shots.rs:125-158); a dq_plan extends that reuse
 * across calls and is what device-timed benchmarks drive.  A run starts from
 * |0...0>, applies every operation and, for a circuit ending in measurements,
 * draws `shots` terminal samples with the per-shot ChaCha8 streams of
 * shots.rs:153-158.  Kernel-class statistics use the dq_kernel_class order. */
typedef struct dq_plan dq_plan;
typedef enum dq_kernel_class {
    DQ_K_GATE1Q = 0,
    DQ_K_CONTROLLED = 1,
    DQ_K_DIAGONAL = 2,
    DQ_K_SWAP = 3,
    DQ_K_DENSE = 4,
    DQ_K_MEASURE = 5,
    DQ_K_TILE = 6,
    DQ_K_FUSED = 7,
    DQ_K_SAMPLE = 8,
    DQ_K_NORM = 9, /* FP64 norms and rescaling between fused passes */
    DQ_K_NUM_CLASSES = 10
} dq_kernel_class;
DQ_API int dq_plan_create(dq_sim* sim, const char* json, size_t json_len, uint64_t shots, dq_plan** out);
/* One run; *device_ms is the CUDA-event time on the engine stream.  With
 * record != 0 every launch is bracketed by events for dq_plan_stats.  A plan
 * created with shots > 0 samples at the end of each run; its complex64 fused
 * form then skips the FP64 rescale after the last fused pass (sampling
 * divides by the total), so its final state keeps that pass's rounding of
 * the norm (~1e-7). */
DQ_API int dq_plan_run(dq_plan* p, int record, double* device_ms);
/* Per kernel class of the last recorded run: milliseconds, kernel launches and
 * algorithmic bytes (arrays of DQ_K_NUM_CLASSES entries). */
DQ_API int dq_plan_stats(const dq_plan* p, double* ms, uint64_t* launches, double* bytes);
DQ_API int dq_plan_info(const dq_plan* p, uint64_t* num_qubits, uint64_t* num_ops, double* state_bytes);
DQ_API int dq_plan_statevector(const dq_plan* p, double* out, uint64_t out_len);
DQ_API int dq_plan_samples(const dq_plan* p, uint64_t* out, uint64_t out_len);
/* State fidelity |<a|b>|^2 / (<a|a> <b|b>) and max amplitude error of two
 * plans' final states (same qubit count, any precisions), computed on the
 * device. */
DQ_API int dq_plan_compare(const dq_plan* a, const dq_plan* b, double* fidelity, double* max_abs_err);
DQ_API void dq_plan_free(dq_plan* p);

/* Batched circuits: many circuits of uneven qubit counts, each a unitary
 * prefix followed only by measurements, run in one persistent kernel over
 * (circuit, pass, tile) work items, then sampled with `shots` terminal
 * samples each (per-shot ChaCha8 streams as shots.rs:153-158) and reduced to
 * <Z0 Z1>.  No counterpart in the reference, which runs one circuit per call;
 * each circuit's counts follow the reference's terminal-sampling semantics
 * (shots.rs:93-176).  autotune = 1 times, per qubit count, candidate tile
 * shapes, fusion widths and shared-memory pass depths of the persistent
 * kernel and (complex64, 12 qubits or more) tensor-core fused passes, which
 * run on side streams beside it; autotune = 2 takes the tensor-core fused
 * passes wherever they apply without timing; 0 keeps the default tile shape.
 * A run can replay a captured CUDA graph. */
typedef struct dq_batch dq_batch;
DQ_API int dq_batch_create(dq_sim* sim, const char* const* jsons, const size_t* json_lens, uint64_t count,
                           uint64_t shots, int autotune, dq_batch** out);
DQ_API int dq_batch_run(dq_batch* b, int use_graph, double* device_ms);
DQ_API int dq_batch_counts(const dq_batch* b, uint64_t index, dq_counts** out);
DQ_API int dq_batch_expect_zz(const dq_batch* b, double* out, uint64_t count);
DQ_API int dq_batch_statevector(const dq_batch* b, uint64_t index, double* out, uint64_t out_len);
DQ_API int dq_batch_info(const dq_batch* b, uint64_t* passes, uint64_t* items);
/* One run's work: algorithmic HBM bytes of its passes (each pass reads and
 * writes its circuit's state once), tensor-core f16 FLOPs of the fused blocks,
 * real CUDA-core FLOPs of the tile operations, and how many circuits run as
 * tensor-core fused passes (the rest run in the persistent tile kernel). */
DQ_API int dq_batch_work(const dq_batch* b, double* bytes, double* tensor_flops, double* cuda_core_flops,
                         uint64_t* fused_circuits);
DQ_API void dq_batch_free(dq_batch* b);

/* Learned fusion cost model (no counterpart in the reference): a 16-64-64-1
 * FP32 MLP predicting log device cycles per tile of one tile-local operation
 * from the features written by the engine (kind, width, tile-local qubit
 * positions, fused gate count, work per tile, tile size, precision).
 * Training, gradients and inference run in CUDA kernels of this library.
 * `record` runs a unitary circuit once with per-operation clock64() timing
 * and appends its samples.  Attached to a simulator, the model picks each
 * tile pass's fusion width; a prepared circuit (dq_plan) then times the
 * learned plan against the greedy fixed-width plan, keeps the faster, and
 * logs a rejection when the learned plan is slower.  Detach a model before
 * freeing it. */
typedef struct dq_cost_model dq_cost_model;
#define DQ_MLP_FEATURES 16
#define DQ_MLP_PARAMS 5315 /* 5313 weights and biases + target mean and std */
DQ_API int dq_cost_model_create(int device, uint64_t seed, dq_cost_model** out);
/* Model kinds.  DQ_COST_TILE_OPS: the model above (tile-local operations and
 * tensor-core blocks; picks each pass's fusion width).  DQ_COST_FUSED_PASSES:
 * prices whole tensor-core passes from their tile qubits, block count, gates
 * per block and the state size (log device nanoseconds per tile); attached to
 * a complex64 simulator it picks, among the candidate fused plans of a wider
 * set of spread caps, the one of least predicted time, in place of the
 * hand-fitted pass and spread constants.  A prepared circuit then times that
 * plan against the hand rule's and keeps the faster (rejections logged). */
#define DQ_COST_TILE_OPS 0
#define DQ_COST_FUSED_PASSES 1
DQ_API int dq_cost_model_create_kind(int device, uint64_t seed, int kind, dq_cost_model** out);
DQ_API int dq_cost_model_kind(const dq_cost_model* m, int* kind);
DQ_API void dq_cost_model_free(dq_cost_model* m);
DQ_API int dq_cost_model_add_samples(dq_cost_model* m, const float* features, const float* log_cycles, uint64_t n);
DQ_API int dq_cost_model_record(dq_cost_model* m, dq_sim* sim, const char* json, size_t json_len, uint64_t* added);
DQ_API int dq_cost_model_num_samples(const dq_cost_model* m, uint64_t* n);
DQ_API int dq_cost_model_samples(const dq_cost_model* m, float* features, float* log_cycles, uint64_t n);
DQ_API int dq_cost_model_train(dq_cost_model* m, int epochs, float lr, double* final_mse);
DQ_API int dq_cost_model_predict(const dq_cost_model* m, const float* features, uint64_t n, float* log_cycles);
/* Gradients of the mean squared error over one batch of 1..128 samples (no update). */
DQ_API int dq_cost_model_gradients(const dq_cost_model* m, const float* features, const float* log_cycles, uint64_t n,
                                   float* grads);
DQ_API int dq_cost_model_get_params(const dq_cost_model* m, float* out, uint64_t len);
DQ_API int dq_cost_model_set_params(dq_cost_model* m, const float* in, uint64_t len);
DQ_API int dq_sim_set_cost_model(dq_sim* sim, dq_cost_model* m);
/* The candidate fused plans of a circuit's unitary prefix as JSON text (no
 * counterpart in the reference): per plan its spread cap, the hand rule's
 * cost and its passes; per distinct pass its tile qubits, blocks, gates and
 * DQ_COST_FUSED_PASSES features, with measure != 0 its device milliseconds
 * (one k_fused launch on a complex64 state of the circuit's size on the
 * simulator's device) and with a model its predicted milliseconds.  wide != 0
 * plans the learned planner's wider set of caps.  Free with dq_string_free. */
DQ_API int dq_fused_portfolio(dq_sim* sim, const char* json, size_t json_len, int wide, int measure,
                              const dq_cost_model* model, char** out_text);
/* The DQ_COST_FUSED_PASSES features (DQ_MLP_FEATURES floats) of a fused
 * pass: its 12 ascending tile qubits over one state of num_qubits qubits, its
 * block count and the gates fused into its blocks.  Host-only. */
DQ_API int dq_fused_pass_features(int num_qubits, const int* tile_qubits, int nblocks, int gates, float* out);
/* `count` (1..4096) seeded random fused passes over num_qubits qubits (14..34): random
 * tile qubits (qubits 0 and 1 plus ten drawn uniformly, low- or high-weighted,
 * or as one window) and 1..10 clusters of random one- and two-qubit gates,
 * with features and, with measure != 0, device milliseconds, as JSON text.
 * Training data of the DQ_COST_FUSED_PASSES model. */
DQ_API int dq_fused_random_passes(dq_sim* sim, int num_qubits, uint64_t count, uint64_t seed, int measure,
                                  char** out_text);
/* Planner outcome of a prepared circuit built while a model was attached. */
DQ_API int dq_plan_planner(const dq_plan* p, double* learned_ms, double* greedy_ms, int* used_learned, int* rejected);
/* Arithmetic of one run of the kept plan (no counterpart in the reference):
 * real floating-point operations on CUDA cores (a complex product counts 6, a
 * complex sum 2; FP64 for complex128 states, FP32 for complex64) and the f16
 * tensor-core FLOPs of the fused blocks (three 128 x 64 x 64 products per
 * block and 4096-amplitude tile).  The numerators of the FLOP rooflines. */
DQ_API int dq_plan_flops(const dq_plan* p, double* cuda_core_flops, double* tensor_flops);
/* Passes, CUDA-core tile operations and tensor-core fused blocks of the kept plan. */
DQ_API int dq_plan_shape(const dq_plan* p, uint64_t* passes, uint64_t* tile_ops, uint64_t* fused_blocks);
/* Planner decisions of a simulator, one JSON object per line; free with dq_string_free. */
DQ_API int dq_sim_planner_log(dq_sim* sim, char** out_text);

/* Free and total memory of CUDA device `device`, in bytes (cudaMemGetInfo).
 * No counterpart in the reference; the device backends' resource preflight
 * (ml/circuit.py:201-217 checks host memory for complex128 states) reads it. */
DQ_API int dq_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes);

/* FP64 fused multiply-add throughput of CUDA device `device` in TFLOP/s,
 * measured by a kernel of this library (eight independent FMA chains per
 * thread, several blocks per SM, best of three timed launches).  No
 * counterpart in the reference; it is the denominator of the complex128 tile
 * kernel's FP64 roofline. */
DQ_API int dq_device_fp64_tflops(int device, double* tflops);

/* Host wall time, in seconds, of the phases of the simulator's last
 * simulate_shots call (no counterpart in the reference, whose shots profile
 * records preprocessing, fusion and total times only, simulator.rs:25-37):
 * out[0] parse and validation, [1] compile, [2] statevector allocation,
 * [3] pass planning and gate images, [4] launching the unitary prefix,
 * [5] probability running sums (waits for the prefix to finish), [6] shot
 * draws and their copy to the host, [7] count keys, [8] freeing the call's
 * device buffers, [9] the whole call, [10] allocating the sampling table
 * (host time, before the prefix is launched) and [11] the device time of the unitary
 * prefix (CUDA events around its launches).  Terminal sampling fills every
 * phase; trajectories fill 0, 1 and 9. */
#define DQ_CALL_PHASES 12
DQ_API int dq_sim_last_call_phases(dq_sim* sim, double* out, uint64_t n);

/* Measure without allocating.  No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc -- hosts whose device memory belongs to
 * their own budgeted allocator and that forbid side allocations, and
 * latency-bound loops that cannot afford the device-wide synchronisation an
 * allocation or a free may cause.  It measures `qubit` of each of
 * `num_states` states of 2^num_qubits amplitudes stored back to back at
 * `states` (the caller's device memory, complex128 or complex64 by
 * `precision`), drawing from ChaCha8 stream seeds[i] at draw draw_index[i]
 * (the per-trajectory streams of shots.rs:224), collapses each state in place
 * (reset != 0 also returns the qubit to |0>) and writes each outcome to host
 * memory outcomes[i].  It calls no cudaMalloc, cudaFree or allocating
 * library routine: its scratch is a fixed 256 KiB __device__ array that
 * every GPU loading this library holds until exit, looked up on the first
 * call on each device.  Requests whose scratch would exceed 256 KiB (about
 * 15 states of 22+ qubits, thousands of small states) fail with
 * DQ_VALUE_ERROR.  All calls share that array: calls whose GPU work overlaps
 * race on it.  The work runs on the legacy default stream and the call
 * returns after it has finished; the legacy stream does not wait for
 * non-blocking streams, so work that writes `states` on another stream must
 * be synchronised before the call.  A state whose norm is zero or not finite
 * is left unchanged with outcomes[i] = -1 and the call returns
 * DQ_RUNTIME_ERROR; the other states of that call are measured and collapsed
 * all the same, with their outcomes in outcomes[]. */
DQ_API int dq_measure_noalloc(void* states, int precision, uint64_t num_states, uint64_t num_qubits, uint64_t qubit,
                              int reset, const uint64_t* seeds, const uint64_t* draw_index, int* outcomes);

/* Dense blocks of the P-block backend on the device.  The reference's
 * P-block model (src/distributed/pblock/model.rs) holds the state as
 * independent dense blocks and runs every gate, merge and measurement on one
 * block with the src/engine.rs kernels; these entry points are the calls it
 * makes, on blocks the caller keeps in device memory (2^num_qubits complex128
 * or complex64 amplitudes by the context's precision, little-endian in the
 * block's local qubits, qubits[0] the MSB of a matrix or probability index).
 * A context owns a non-blocking stream: its calls run in order on it,
 * asynchronously except dq_block_measure (which returns the outcome) and
 * dq_blocks_sync.  It does not wait for other streams, so work that writes a
 * block elsewhere must be synchronised before the call, and a block must stay
 * allocated until the context's stream has used it.  The block bookkeeping
 * (which qubits a block holds, when to merge) stays with the caller, as in
 * model.rs. */
typedef struct dq_blocks dq_blocks;
DQ_API int dq_blocks_create(int device, int precision, dq_blocks** out);
DQ_API void dq_blocks_destroy(dq_blocks* ctx);
DQ_API int dq_blocks_sync(dq_blocks* ctx);
/* engine::apply_one_qubit (model.rs:322-324): matrix is 2x2 row-major complex
 * as 8 doubles (re, im); controls are (qubit, value) pairs. */
DQ_API int dq_block_apply_one_qubit(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t target,
                                    const double* matrix, const uint64_t* ctl_qubits, const uint8_t* ctl_values,
                                    size_t num_controls);
/* engine::apply_x (model.rs:320). */
DQ_API int dq_block_apply_x(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t target,
                            const uint64_t* ctl_qubits, const uint8_t* ctl_values, size_t num_controls);
/* engine::apply_swap (model.rs:370). */
DQ_API int dq_block_apply_swap(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t a, uint64_t b,
                               const uint64_t* ctl_qubits, const uint8_t* ctl_values, size_t num_controls);
/* engine::apply_diagonal (model.rs:415): k <= 5 qubits, 2^k complex entries as doubles. */
DQ_API int dq_block_apply_diagonal(dq_blocks* ctx, void* state, uint64_t num_qubits, const uint64_t* qubits, size_t k,
                                   const double* diagonal);
/* engine::DenseLayout::apply (model.rs:429): k <= 5 qubits, row-major 2^k x 2^k complex. */
DQ_API int dq_block_apply_dense(dq_blocks* ctx, void* state, uint64_t num_qubits, const uint64_t* qubits, size_t k,
                                const double* matrix);
/* engine::measure_qubit (model.rs:484-486) with the caller's draw in [0, 1):
 * outcome = draw < p1 / (p0 + p1), the block collapsed and renormalised. */
DQ_API int dq_block_measure(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t qubit, double draw,
                            int* outcome);
/* The merge of two blocks (model.rs:199-248): out[i * 2^left_qubits + j] =
 * left[j] * right[i], the left block's qubits becoming the low ones. */
DQ_API int dq_block_merge(dq_blocks* ctx, const void* left, uint64_t left_qubits, const void* right,
                          uint64_t right_qubits, void* out);
/* engine::marginal_probs over `qubits` (k = 0: every amplitude's |a|^2) into
 * device memory `out` (2^k doubles). */
DQ_API int dq_block_probabilities(dq_blocks* ctx, const void* state, uint64_t num_qubits, const uint64_t* qubits,
                                  size_t k, double* out);
/* The running sums of a block's squared magnitudes that P-block sampling
 * draws from (model.rs:583-608), into device memory `out` (2^num_qubits doubles). */
DQ_API int dq_block_running_sums(dq_blocks* ctx, const void* state, uint64_t num_qubits, double* out);

/* Host-only helpers (no device work): parse, validate and compile a circuit
 * exactly as read_circuit + compile do (simulator.rs:204-211,
 * execution.rs:368-416), returning the operation list as JSON text with
 * doubles as 16-hex-digit bit patterns.  Free the text with dq_string_free. */
DQ_API int dq_compile_dump(const char* json, size_t json_len, char** out_text);
/* Host-only: the shared-memory tile plan of the circuit's unitary operations
 * (tile qubits, tile-local operations, matrix pool) as JSON text.  No
 * counterpart in the reference; it exposes the planner for inspection. */
DQ_API int dq_tile_plan_dump(const char* json, size_t json_len, int tile_qubits, int fusion_width, char** out_text);
/* Host-only: the tensor-core fused plan (12-qubit passes of 32x32 blocks: layout
 * tables, f16 hi/lo gate images and each pass's TMA box plan) as JSON text.  No
 * counterpart in the reference. */
DQ_API int dq_fused_plan_dump(const char* json, size_t json_len, char** out_text);
/* Failure-path testing of the fused tensor-core kernel (no counterpart in the
 * reference): from the next launch on, gate images of fused steps >=
 * withhold_step are never fetched, and every bounded wait of the kernel gives
 * up after wait_ms milliseconds (<= 0: the default, about 2 s).  A pass that
 * runs out sets the device error flag and the call raises DQ_RUNTIME_ERROR;
 * the context stays usable.  withhold_step = UINT64_MAX restores normal
 * operation.  Process-wide; not for concurrent use. */
DQ_API int dq_debug_fused_fault(uint64_t withhold_step, double wait_ms);
DQ_API void dq_string_free(char* s);

#ifdef __cplusplus
}
#endif

#endif /* DQSIM_SV_H */

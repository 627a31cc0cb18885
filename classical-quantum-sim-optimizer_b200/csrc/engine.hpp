// Device runtime: memory, batches of states and the operation executor.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "compile.hpp"
#include "kernels.hpp"
#include "phased.hpp"
#include "tile.hpp"

namespace dq {

void cuda_check(cudaError_t e, const char* what);

// Runs fn(0) .. fn(count - 1) on the calling thread and up to 15 pooled host
// workers; the first exception a call throws is rethrown here after every
// item that started has finished (items not yet started are skipped).
void parallel_for(size_t count, const std::function<void(size_t)>& fn);

// Owning device allocation.  Allocation failure is a MemoryError, as the
// reference reports a failed statevector reservation (shots.rs:33-41).
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;  // set: stream-ordered block from the engine's memory pool
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }
    void alloc(size_t b, const char* what);
    // Stream-ordered allocation from the engine's pool on this device: the
    // block returns to the pool when released, in order on stream s, so the
    // next large buffer of the same size costs no driver mapping.
    void alloc_on(size_t b, cudaStream_t s, const char* what);
    void ensure(size_t b, const char* what) {
        if (b > bytes) alloc(b, what);
    }
    void ensure_on(size_t b, cudaStream_t s, const char* what) {
        if (b > bytes) alloc_on(b, s, what);
    }
    void release();
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// One CUDA device + stream used by a simulator and the results it returns.
struct Device {
    int ordinal = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;  // serialises calls on the simulator and its results
    explicit Device(int ordinal);
    ~Device();
    void sync();
    void activate() const;
};

// W states of n qubits plus per-state classical bits and measurement scratch.
struct StateBatch {
    DevMem amps, cbits, seeds, draws, outcome, scale, partial, err;
    int n = 0;
    uint64_t W = 0, ncb = 0;
    int cwords = 1;
    bool c64 = false;
    // With a stream, the statevector comes from the stream-ordered pool.
    void allocate(int n, uint64_t W, uint64_t ncb, bool c64, cudaStream_t pool_stream = nullptr);
    k::Batch view(cudaStream_t s, uint64_t W_active) const;
    size_t amp_bytes() const { return size_t(1) << n; }
};

struct ProfileAcc {
    uint64_t oq_calls = 0, nq_calls = 0, mq_calls = 0;
    double oq_time = 0, nq_time = 0, mq_time = 0;
};

// Kernel classes timed by the event recorder (bench and roofline).
enum KernelClass : int {
    kcGate1q = 0,    // uncontrolled 2x2 on pairs
    kcControlled,    // controlled 2x2 / X on pairs
    kcDiagonal,
    kcSwap,
    kcDense,
    kcMeasure,
    kcTile,          // shared-memory multi-gate pass
    kcFused,         // tensor-core fused-block pass
    kcSample,
    kcNorm,          // FP64 norms and rescaling between fused passes
    kcNumClasses
};
const char* kernel_class_name(int c);

// Records a CUDA event pair around each launch of the stream, tagged with a
// kernel class and the launch's algorithmic bytes; durations are read after
// the stream drains.
class EventRecorder {
  public:
    explicit EventRecorder(cudaStream_t s) : stream_(s) {}
    ~EventRecorder();
    // `kernels`: launches inside the bracket.
    void begin(int cls, double bytes, int kernels = 1);
    void end();
    // Totals per class: milliseconds, launches, algorithmic bytes.
    void collect(double* ms, uint64_t* launches, double* bytes);

  private:
    struct Rec {
        int cls;
        double bytes;
        cudaEvent_t a, b;
        int kernels;
    };
    cudaStream_t stream_;
    std::vector<Rec> recs_;
    std::vector<cudaEvent_t> pool_;
    cudaEvent_t take();
};

// How an executor lowers unitary runs.
struct ExecConfig {
    bool tiled = false;  // shared-memory tile passes for unconditioned unitary runs
    int tile_m = 12;     // tile qubits
    int fuse = 2;        // widest fused dense operation inside a pass
    int seeds = 6;       // planner candidates per pass
    int n = 0;           // qubits of the state the plan runs on
    bool c64 = false;
    const CostModel* model = nullptr;  // learned fusion-width choice per pass
    bool fused = false;  // complex64: 5-qubit blocks on tcgen05 (12-qubit tiles)
    // Learned pass-cost model: picks the fused plan of least predicted time
    // from the wide portfolio (kCostFusedPasses models only).
    const CostModel* pass_model = nullptr;
    // Tile passes run in register phases (phased.hpp).  Passes planned with a
    // tile-op cost model keep one operation per sweep, the form that model's
    // per-operation costs were recorded on.
    bool phased = true;
};

// How the fused plan of a segment was chosen: the portfolio's caps, the hand
// rule's cost of each plan and its choice, and, with a pass-cost model, the
// predicted milliseconds of each plan and the model's choice.
struct FusedPlanChoice {
    std::vector<int> caps;
    std::vector<double> rule_cost, predicted_ms;
    std::vector<size_t> passes, blocks;
    size_t rule_choice = 0, chosen = 0;
};

// A compiled operation list lowered to launch descriptors, with every matrix
// uploaded once into a device pool.  Per-gate steps are one launch per
// operation (the reference-faithful plain form); tiled steps run a planned
// shared-memory pass over every tile of the state.
class Executor {
  public:
    Executor(const std::vector<Operation>& ops, size_t begin, size_t end, const ExecConfig& cfg = ExecConfig());
    // Launch every step on the batch (asynchronously unless `profile`).
    // `normalize` false: when the last step is a fused tensor-core pass, its
    // FP64 norm and rescale are left out (the state keeps the pass's rounding
    // of the norm, ~1e-7); for callers that only sample, which divides by the
    // total probability anyway.
    // `from_basis`: every state of the batch is |0...0> on entry; a first step
    // that is a fused pass then builds its input tiles itself (the caller
    // need not write the state first: starts_with_fused_pass()).
    void run(const k::Batch& b, ProfileAcc* profile, EventRecorder* rec = nullptr, bool normalize = true,
             bool from_basis = false);
    bool starts_with_fused_pass() const { return !steps_.empty() && steps_[0].fused >= 0; }
    // Uploads the matrix pools and sizes the scratch a run over batches like
    // `b` needs, so that later runs allocate nothing and copy nothing from the
    // host (they can then be captured into a CUDA graph).
    void prepare(const k::Batch& b);
    size_t steps() const { return steps_.size(); }
    // Algorithmic bytes one step moves for a batch (the roofline numerator).
    double step_bytes(size_t i, const k::Batch& b) const;
    // Arithmetic of one run over a batch, for the FLOP rooflines: real
    // floating-point operations on CUDA cores (a complex product counts 6, a
    // complex sum 2; FP64 for complex128 states, FP32 for complex64) and the
    // f16 tensor-core FLOPs the fused blocks issue.
    void arith_flops(const k::Batch& b, double* cuda_core, double* tensor) const;

    size_t passes() const { return passes_.size() + fused_.size(); }
    size_t fused_blocks() const { return fused_blocks_host_.size(); }
    size_t raw_ops_in_passes() const;
    const std::vector<int>& chosen_widths() const { return widths_; }
    const std::vector<FusedPlanChoice>& fused_choices() const { return fused_choices_; }
    size_t tile_ops() const { return tile_ops_host_.size(); }
    // Times every pass (CUDA events), shares each pass's time among its
    // operations by their clock64 cycles or equally among its tensor-core
    // blocks, and appends (features, log picoseconds per tile) samples.  Fused
    // passes are also timed on CUDA cores at each fusion width, so that the
    // planner can compare the two executors pass by pass.
    void record_costs(const k::Batch& b, std::vector<float>& X, std::vector<float>& y);

  private:
    struct Step {
        int pass = -1;   // >= 0: a tile pass (index into passes_)
        int fused = -1;  // >= 0: a tensor-core fused pass (index into fused_)
        Operation::Type type;
        int target = 0, a = 0, b = 0;
        std::vector<k::Ctl> controls;
        double2 u[4] = {};
        std::vector<int> qubits;
        std::vector<double2> diag;
        size_t pool_offset = 0;  // Dense: index into the matrix pool (double2 units)
        int64_t cbit = -1;
        dev::CondList cond{};
        std::vector<Condition> host_conds;
        int category = 0;  // profile bucket as in execution.rs:297-347
    };
    std::vector<Step> steps_;
    std::vector<double2> pool_host_;
    std::vector<TilePass> passes_;
    std::vector<TileOp> tile_ops_host_;
    std::vector<FusedPass> fused_;
    std::vector<TilePass> fused_src_;  // each fused pass's tile qubits and raw operations
    std::vector<FusedBlock> fused_blocks_host_;
    std::vector<uint16_t> upool_host_;
    std::vector<std::vector<uint4>> phase_blocks_;  // per phased pass (host copies: launch arguments)
    std::vector<uint4> phase_words_host_;           // the same blocks back to back (device copy)
    DevMem pool_, tile_ops_, fused_blocks_, upool_, norm_tiles_, norm_states_, phase_words_;
    bool uploaded_ = false;
    ExecConfig cfg_;
    std::vector<int> widths_;
    std::vector<FusedPlanChoice> fused_choices_;
    void upload(cudaStream_t stream);
    void lower(const Operation& op, std::vector<Condition>& conds);
    void lower_segment(const std::vector<Operation>& ops, size_t begin, size_t end);
    void attach_phases(TilePass& p);
};

}  // namespace dq

// Many circuits of uneven qubit counts in one CUDA graph.
//
// Every circuit is compiled and planned on the host.  Circuits planned as
// CUDA-core tile passes run in one persistent kernel over a queue of work
// items (circuit, pass, tile) ordered pass level by pass level; an item of
// pass p waits, with a bounded spin, until its circuit's counter shows every
// tile of pass p-1 written back.  Complex64 circuits of 12 or more qubits
// whose shape is tensor-core fused passes run those passes (k_fused) on side
// streams forked from the main stream, longest first onto the least loaded
// stream, beside the persistent kernel.  Terminal sampling (FP64
// probabilities, segmented CDF, per-shot ChaCha8 draws) and the <Z0 Z1>
// expectation of every circuit follow as batched kernels once every stream has
// joined.  The whole sequence is captured once in a CUDA graph and replayed.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "simulator.hpp"
#include "tile.hpp"

namespace dq {

// How the circuits of one qubit count run.  fuse 5 (complex64, >= 12 qubits):
// tensor-core fused passes; otherwise CUDA-core tile passes of tile_m qubits
// with operations fused to `fuse` qubits and at most `depth` operations per
// shared-memory pass (0: no limit).
struct BatchShape {
    int tile_m = 0, fuse = 0, depth = 0;
};

struct BatchTuning {
    int tile_m = 0;   // 0: per qubit count from `per_n`, else the precision's default
    int fuse = 0;
    int depth = 0;
    std::map<uint64_t, BatchShape> per_n;
};

class BatchRun {
  public:
    BatchRun(Simulator& sim, const std::vector<std::string>& circuits, uint64_t shots, const BatchTuning& tuning);
    ~BatchRun();
    // One full batch; returns device milliseconds.  use_graph replays a
    // captured CUDA graph (captured on first use).
    double run(bool use_graph);
    size_t size() const { return circuits_.size(); }
    // Counts of circuit i over its classical register (measured qubits, last write wins).
    std::unordered_map<std::string, uint64_t> counts(size_t i) const;
    std::vector<double> expect_zz() const;
    void statevector(size_t i, double* out) const;
    uint64_t num_qubits(size_t i) const { return circuits_[i].n; }
    size_t passes() const;
    uint64_t items() const { return total_items_; }
    // Algorithmic HBM bytes of one run's passes (every pass reads and writes
    // its circuit's state once) and the arithmetic: tensor-core f16 FLOPs of
    // the fused blocks, real CUDA-core FLOPs of the tile operations.
    void work(double* bytes, double* tensor_flops, double* cuda_core_flops) const;
    size_t fused_circuits() const;
    int error_flag() const;

    struct PassRec {  // device record of one (circuit, pass)
        uint64_t state_off;    // amplitude offset of the circuit's state
        uint64_t item_begin;   // first queue index of this pass
        uint64_t wait_count;   // tiles of earlier passes of the circuit that must be done
        int circuit;
        int n, m;
        int op_begin, nops;
        int q[20];
    };

  private:
    struct Circ {
        uint64_t n = 0, ncb = 0, state_off = 0, seed = 0;
        std::vector<std::pair<uint64_t, uint64_t>> cbit_map;  // (cbit, shift in sampled index)
        std::vector<uint64_t> sample_qubits;                  // descending
        bool full_register = true;
        int tile_m = 12, fuse = 2, depth = 0;
        std::unique_ptr<Executor> fused;  // tensor-core passes on a side stream
        int stream = 0;                   // its side stream
    };
    std::shared_ptr<Device> dev_;
    bool c64_ = true;
    uint64_t shots_ = 0;
    std::vector<Circ> circuits_;
    std::vector<PassRec> pass_recs_;
    std::vector<TileOp> ops_host_;
    std::vector<double2> pool_host_;
    uint64_t total_items_ = 0, total_amps_ = 0;
    int max_m_ = 0;
    DevMem amps_, recs_, ops_, pool_, done_, head_, err_, probs_, tmp_, circ_off_, circ_of_tile_, samples_, zz_part_,
        seeds_;
    cudaGraphExec_t graph_ = nullptr;
    std::vector<cudaStream_t> side_;
    std::vector<cudaEvent_t> join_;
    cudaEvent_t fork_ = nullptr;
    double tile_bytes_ = 0, tile_flops_ = 0;
    void enqueue();
    k::Batch circuit_view(const Circ& c, cudaStream_t s) const;
};

// Autotuner: picks tile qubits and fusion width per qubit count by timing
// candidate plans of a representative circuit on the device; results are
// cached for the process.
struct TuneResult {
    int tile_m, fuse, depth;
    double ms;
};
TuneResult autotune_tile(Simulator& sim, const std::string& circuit_json, bool c64);

}  // namespace dq

// Many circuits of uneven qubit counts in one persistent launch.
//
// Every circuit is compiled and planned into shared-memory tile passes on the
// host.  The device runs one persistent kernel over a queue of work items
// (circuit, pass, tile) ordered pass level by pass level; an item of pass p
// waits, with a bounded spin, until its circuit's counter shows every tile of
// pass p-1 written back.  Terminal sampling (FP64 probabilities, segmented
// CDF, per-shot ChaCha8 draws) and the <Z0 Z1> expectation of every circuit
// follow as batched kernels.  The whole sequence is captured once in a CUDA
// graph and replayed.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "simulator.hpp"
#include "tile.hpp"

namespace dq {

struct BatchTuning {
    int tile_m = 0;   // 0: per qubit count from `per_n`, else the precision's default
    int fuse = 0;
    std::map<uint64_t, std::pair<int, int>> per_n;  // qubits -> (tile qubits, fusion width)
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
    size_t passes() const { return pass_recs_.size(); }
    uint64_t items() const { return total_items_; }
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
        int tile_m = 12, fuse = 2;
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
    void enqueue();
};

// Autotuner: picks tile qubits and fusion width per qubit count by timing
// candidate plans of a representative circuit on the device; results are
// cached for the process.
struct TuneResult {
    int tile_m, fuse;
    double ms;
};
TuneResult autotune_tile(Simulator& sim, const std::string& circuit_json, bool c64);

}  // namespace dq

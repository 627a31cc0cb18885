// A prepared circuit: parsed, validated, compiled and lowered once, with its
// state and sampling buffers resident on the device, then run many times.
//
// This is the reuse the reference applies inside one simulate_shots call (one
// compiled plan and one prefix evolution shared by every shot,
// src/monolithic/statevector/shots.rs:125-158), exposed across calls so that
// device time can be measured without host work in the timed region.
#pragma once

#include <memory>
#include <vector>

#include "simulator.hpp"

namespace dq {

class Plan {
  public:
    Plan(Simulator& sim, const char* json, size_t len, uint64_t shots);
    // One full run: |0>, every operation, then terminal sampling when the
    // circuit ends in measurements.  Returns device milliseconds (CUDA events
    // on the engine stream).  With `record`, per-kernel-class events are kept.
    double run(bool record);
    void stats(double* ms, uint64_t* launches, double* bytes) const;
    void statevector(double* out) const;
    void samples(uint64_t* out) const;
    uint64_t num_qubits() const { return n_; }
    uint64_t num_ops() const { return ops_.size(); }
    uint64_t shots() const { return shots_; }
    double state_bytes() const;
    // |<this|other>|^2 and max |a_i - b_i| of the two final states, on the device.
    void compare(const Plan& other, double* fidelity, double* max_abs_err) const;
    // Learned-vs-greedy planner outcome (zeros when no cost model was attached).
    void planner(double* learned_ms, double* greedy_ms, int* used_learned, int* rejected) const {
        *learned_ms = learned_ms_;
        *greedy_ms = greedy_ms_;
        *used_learned = used_learned_ ? 1 : 0;
        *rejected = rejected_ ? 1 : 0;
    }
    // Arithmetic of one run's operations (Executor::arith_flops).
    void flops(double* cuda_core, double* tensor) const {
        ex_->arith_flops(st_.view(nullptr, 1), cuda_core, tensor);
    }
    size_t passes() const { return ex_ ? ex_->passes() : 0; }
    size_t tile_ops() const { return ex_ ? ex_->tile_ops() : 0; }
    size_t fused_blocks() const { return ex_ ? ex_->fused_blocks() : 0; }
    // Appends per-operation cost samples of one recorded run.
    void record_costs(std::vector<float>& X, std::vector<float>& y);

  private:
    std::shared_ptr<Device> dev_;
    Options opt_;
    uint64_t n_ = 0, ncb_ = 0, shots_ = 0, seed_ = 0;
    std::vector<Operation> ops_;
    size_t prefix_end_ = 0;
    bool terminal_ = false;
    std::vector<uint64_t> sample_qubits_;
    StateBatch st_;
    std::unique_ptr<Executor> ex_;
    DevMem cdf_, tmp_, idx_, scalar_;
    double ms_[kcNumClasses] = {}, bytes_[kcNumClasses] = {};
    uint64_t launches_[kcNumClasses] = {};
    double learned_ms_ = 0, greedy_ms_ = 0;
    bool used_learned_ = false, rejected_ = false;
};

}  // namespace dq

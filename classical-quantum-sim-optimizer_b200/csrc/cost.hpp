// Learned cost model for the fusion planner.
//
// A 16 -> 64 -> 64 -> 1 MLP (ReLU, FP32) predicts the log of the device time
// (picoseconds per tile of the pass) one candidate costs: a CUDA-core
// tile-local operation, from its kind, width, the tile-local positions of its
// qubits (stride and bank-conflict class), how many gates were fused into it,
// its work per tile and the tile size; or a 5-qubit tensor-core block, from
// its qubit positions, gate count and the pass's block count (which carries
// the pass's load and store).  It is trained on timings the engine records
// itself: each pass is timed with CUDA events and its time is shared among
// its operations by their clock64() cycles (an instrumented tile pass reads
// the clock around every operation) or equally among its blocks.  Training
// and inference are CUDA kernels written here: one CTA runs mini-batch
// forward, backward and Adam steps; inference is one thread per candidate.
// The planner asks it, per pass, which fusion width (CUDA cores) or the
// tensor-core blocks is cheapest; the greedy plan stays the fallback and the
// judge.
//
// A model of the second kind (kCostFusedPasses) prices whole tensor-core
// passes instead: from a pass's tile qubits (where they sit in the state, the
// hand rule's run and spread ingredients, its TMA box count), its block count
// and gates per block and the state size, it predicts the log of the pass's
// device time per tile.  Trained on passes the engine times itself (every
// distinct pass of the candidate plans of recorded circuits, and seeded
// random passes), it chooses which of the candidate fused plans to run in
// place of the hand-fitted pass and spread constants; the hand rule's plan is
// the fallback, and every learned plan is timed against it.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "tile.hpp"

namespace dq {

constexpr int kMlpF = 16;   // features
constexpr int kMlpH = 64;   // hidden width
constexpr int kMlpB = 128;  // training mini-batch
constexpr int kMlpParams = kMlpH * kMlpF + kMlpH + kMlpH * kMlpH + kMlpH + kMlpH + 1;

// Features of one tile-local operation in a pass of m tile qubits.
void tile_op_features(const TileOp& op, int m, bool c64, float* out);
// Features of one tensor-core block (local qubit mask, fused gates) in a
// fused pass of `nblocks` blocks.
void fused_block_features(int gates, uint32_t local_mask, int nblocks, float* out);
// Features of one whole fused pass (kCostFusedPasses): its 12 tile qubits
// over `states` states of n qubits, its block count and gates.
void fused_pass_features(int n, uint64_t states, const std::vector<int>& tile_qubits, int nblocks, int gates,
                         float* out);

enum CostKind : int {
    kCostTileOps = 0,      // CUDA-core tile operations and tensor-core blocks (fusion width per pass)
    kCostFusedPasses = 1,  // whole tensor-core passes (which candidate fused plan runs)
};

class CostModel {
  public:
    CostModel(int device, uint64_t seed, int kind = kCostTileOps);
    int kind() const { return kind_; }
    ~CostModel();
    void add_samples(const float* X, const float* y, size_t n);
    size_t num_samples() const { return y_.size(); }
    void copy_samples(float* X, float* y) const {
        std::lock_guard<std::mutex> lk(mu_);
        std::copy(X_.begin(), X_.end(), X);
        std::copy(y_.begin(), y_.end(), y);
    }
    // Adam on the log targets; returns the final epoch's mean squared error.
    double train(int epochs, float lr);
    void predict(const float* X, size_t n, float* out) const;
    // Gradients of the mean squared error for one batch (n <= kMlpB), no update.
    void gradients(const float* X, const float* y, size_t n, float* grads) const;
    void get_params(float* out) const;
    void set_params(const float* in);
    bool trained() const { return trained_; }
    // Sum of the predicted costs of a list of operations (one device call).
    double predict_ops(const std::vector<TileOp>& ops, int m, bool c64) const;
    // Sum of the predicted costs of a fused pass's blocks.
    double predict_fused(const FusedPass& p) const;
    // Predicted device milliseconds of each distinct pass of a fused
    // portfolio over `states` states (kCostFusedPasses), and of each plan.
    std::vector<double> predict_passes_ms(const FusedPortfolio& pf, uint64_t states) const;
    std::vector<double> predict_plans_ms(const FusedPortfolio& pf, uint64_t states) const;
    int device() const { return device_; }

  private:
    int device_;
    int kind_ = kCostTileOps;
    bool trained_ = false;
    std::vector<float> X_, y_;
    void* params_ = nullptr;  // device: params, adam m, adam v
    cudaStream_t stream_ = nullptr;
    mutable std::mutex mu_;
};

}  // namespace dq

// Dense blocks of the P-block backend on the device (see blocks.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "engine.hpp"

namespace dq {

class BlockContext {
  public:
    BlockContext(int device, bool c64);
    ~BlockContext();
    BlockContext(const BlockContext&) = delete;
    BlockContext& operator=(const BlockContext&) = delete;
    bool c64() const { return c64_; }
    // m: 2x2 row-major complex matrix as 8 doubles (re, im); is_x swaps the pair.
    void apply_one_qubit(void* state, uint64_t n, uint64_t target, const double* m, const uint64_t* ctl_qubits,
                         const uint8_t* ctl_values, size_t num_controls, bool is_x);
    void apply_swap(void* state, uint64_t n, uint64_t a, uint64_t b, const uint64_t* ctl_qubits,
                    const uint8_t* ctl_values, size_t num_controls);
    // qubits[0] is the MSB of the diagonal / matrix index.
    void apply_diagonal(void* state, uint64_t n, const uint64_t* qubits, size_t k, const double* diagonal);
    void apply_dense(void* state, uint64_t n, const uint64_t* qubits, size_t k, const double* matrix);
    // Collapses the block and returns the outcome (synchronises the stream).
    int measure(void* state, uint64_t n, uint64_t qubit, double draw);
    void merge(const void* left, uint64_t nl, const void* right, uint64_t nr, void* out);
    // Marginal probabilities over `qubits` (qubits[0] MSB); k = 0: every amplitude's |a|^2.
    void probabilities(const void* state, uint64_t n, const uint64_t* qubits, size_t k, double* out);
    // Inclusive running sums of the block's squared magnitudes (2^n doubles).
    void running_sums(const void* state, uint64_t n, double* out);
    void sync();

  private:
    int device_;
    bool c64_;
    cudaStream_t stream_ = nullptr;
    DevMem outcome_, scale_, partial_, cbits_, err_, mat_, tmp_;
    k::Batch batch(void* state, uint64_t n);
};

}  // namespace dq

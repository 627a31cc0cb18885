// Device runtime: memory, batches of states and the operation executor.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "compile.hpp"
#include "kernels.hpp"

namespace dq {

void cuda_check(cudaError_t e, const char* what);

// Owning device allocation.  Allocation failure is a MemoryError, as the
// reference reports a failed statevector reservation (shots.rs:33-41).
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }
    void alloc(size_t b, const char* what);
    void ensure(size_t b, const char* what) {
        if (b > bytes) alloc(b, what);
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
    void allocate(int n, uint64_t W, uint64_t ncb, bool c64);
    k::Batch view(cudaStream_t s, uint64_t W_active) const;
    size_t amp_bytes() const { return size_t(1) << n; }
};

struct ProfileAcc {
    uint64_t oq_calls = 0, nq_calls = 0, mq_calls = 0;
    double oq_time = 0, nq_time = 0, mq_time = 0;
};

// A compiled operation list lowered to launch descriptors, with every dense
// matrix uploaded once into a device pool.  `fuse_1q_runs` is off for the
// reference-faithful per-gate form.
class Executor {
  public:
    Executor(const std::vector<Operation>& ops, size_t begin, size_t end);
    // Launch every step on the batch (asynchronously unless `profile`).
    void run(const k::Batch& b, ProfileAcc* profile);
    size_t steps() const { return steps_.size(); }

  private:
    struct Step {
        Operation::Type type;
        int target = 0, a = 0, b = 0;
        std::vector<k::Ctl> controls;
        double2 u[4];
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
    DevMem pool_;
    bool uploaded_ = false;
    void lower(const Operation& op, std::vector<Condition>& conds);
};

}  // namespace dq

// StatevectorSimulator / SimulationResult semantics on the device.
//
// Mirrors src/monolithic/statevector/simulator.rs:214-372 (constructor
// checks, simulate, simulate_shots, result queries) and
// src/monolithic/statevector/shots.rs:22-260 (budget arithmetic, terminal
// sampling vs trajectories, per-shot ChaCha8 streams, last-write cbit mapping).
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "compile.hpp"
#include "engine.hpp"

namespace dq {

enum class Precision { C128 = 0, C64 = 1 };

struct Options {
    bool has_seed = false;
    uint64_t seed = 0;
    bool profile = false;
    uint64_t max_memory_mb = 1024;
    bool has_max_parallel_shots = false;
    uint64_t max_parallel_shots = 0;
    bool sample_terminal = true;
    Precision precision = Precision::C128;
    int device = 0;
    int execution = 0;      // 0 auto (tiled), 1 per-gate, 2 tiled
    int tile_qubits = 0;    // 0: 12 for complex128, 13 for complex64
    int fusion_width = 0;   // 0: 2
};

// Executor configuration for a state of n qubits under these options.
ExecConfig exec_config(const Options& o, uint64_t n, bool force_per_gate = false, const CostModel* model = nullptr);

struct ShotOutput {
    std::unordered_map<std::string, uint64_t> counts;
    // Terminal sampling fills these instead of `counts`: distinct keys of
    // key_width characters back to back, one count each.
    std::string flat_keys;
    std::vector<uint64_t> flat_counts;
    uint64_t key_width = 0;
    std::vector<double> shot_times;
    std::string strategy;
    uint64_t parallel_shots = 0;
    uint64_t working_bytes = 0;
    uint64_t prefix_ops = 0;
};

// Host wall time of the phases of the last simulate_shots call on a
// simulator, in seconds (terminal sampling fills every phase; trajectories
// fill parse, compile and total).  Phase order of dq_sim_last_call_phases.
enum CallPhase : int {
    kPhParse = 0,   // JSON parse and validation
    kPhCompile,     // operation lowering and 1q fusion
    kPhState,       // statevector allocation and |0...0> (enqueued)
    kPhPlan,        // pass planning, fused blocks and gate images
    kPhRun,         // uploads and kernel launches of the unitary prefix (enqueued)
    kPhSums,        // probability running sums, waits for the prefix to finish
    kPhSample,      // shot draws and the device-to-host copy of the outcomes
    kPhKeys,        // sorting outcomes into distinct count keys
    kPhRelease,     // freeing the call's device buffers
    kPhTotal,
    kPhTable,         // allocating the sampling table and its scan scratch (before the prefix)
    kPhPrefixDevice,  // device time of the unitary prefix (CUDA events on the simulator's stream)
    kNumCallPhases
};

struct ProfileData {
    bool present = false;
    ProfileAcc acc;
    double total_time = 0;
};

class Result {
  public:
    std::shared_ptr<Device> dev;
    StateBatch state;
    uint64_t n = 0;
    std::vector<uint8_t> cbits;
    ProfileData profile;

    void statevector(double* out_interleaved) const;
    // 2^k doubles; qubits[0] is the MSB of the output index.
    void probabilities(const std::vector<uint64_t>& qubits, double* out) const;
    std::unordered_map<uint64_t, uint64_t> counts(uint64_t shots, const std::vector<uint64_t>& qubits,
                                                  uint64_t seed) const;
    double fidelity(const double* other_interleaved, uint64_t len) const;
    // Amplitudes at the given indices (interleaved re/im), read on the device.
    void amplitudes(const uint64_t* indices, uint64_t count, double* out_interleaved) const;
    // <psi| X^x Z^z |psi> as (re, im), reduced on the device in FP64.
    void pauli_xz(uint64_t x, uint64_t z, double* re, double* im) const;
};

// A circuit text this simulator ran through simulate_shots: its compiled
// operations and, once a terminal-sampling call has planned it, the executor
// of its unitary prefix (passes, fused blocks and gate images on the device).
// A call with the byte-identical text reuses both, skipping parse, validation,
// compilation and planning, which give the same result for the same text.
struct ShotPlan {
    std::string json;
    std::vector<Operation> ops;
    uint64_t n = 0, ncb = 0;
    std::unique_ptr<Executor> prefix;
};

// Device buffers of terminal sampling, kept by a simulator between calls:
// the statevector with its bookkeeping, the sampling table, the scan scratch
// and the drawn outcomes.  A call whose sizes match the previous one's
// allocates nothing.  Allocating them per call from the stream-ordered pool
// cost 50 ms to over 1 s of host time per 8 GiB buffer at 30 qubits: small
// bookkeeping blocks carved from the freed large ones left no whole free
// block, and the pool mapped the memory again.
struct SamplingWorkspace {
    StateBatch st;
    DevMem table, scratch, outcomes;
};

class Simulator {
  public:
    explicit Simulator(const Options& o);
    ~Simulator();
    ShotOutput simulate_shots(const char* json, size_t len, uint64_t shots, bool profile, double* preprocessing,
                              double* fusion);
    std::unique_ptr<Result> simulate(const char* json, size_t len);
    const Options& options() const { return opt_; }
    // Opens the CUDA device on first use.
    std::shared_ptr<Device> ensure_device() {
        std::lock_guard<std::mutex> lk(mu_);
        if (!dev_) dev_ = std::make_shared<Device>(opt_.device);
        return dev_;
    }
    // Learned fusion planner (not owned; detach before the model is freed).
    // Plans cached before it changed no longer apply.
    void set_cost_model(const CostModel* m) {
        std::lock_guard<std::mutex> lk(mu_);
        model_ = m;
        plans_.clear();
    }
    const CostModel* cost_model() const { return model_; }
    // Planner decisions: one JSON object per prepared circuit that compared
    // a learned plan with the greedy one (rejections included).
    void log_planner(const std::string& line) {
        std::lock_guard<std::mutex> lk(mu_);
        planner_log_.push_back(line);
    }
    void last_call_phases(double* out) {
        std::lock_guard<std::mutex> lk(mu_);
        for (int i = 0; i < kNumCallPhases; i++) out[i] = phases_[i];
    }
    std::string planner_log() {
        std::lock_guard<std::mutex> lk(mu_);
        std::string s;
        for (auto& l : planner_log_) s += l + "\n";
        return s;
    }

  private:
    Options opt_;
    uint64_t budget_ = 0;
    std::mutex mu_;
    std::shared_ptr<Device> dev_;
    const CostModel* model_ = nullptr;
    std::vector<std::string> planner_log_;
    double phases_[kNumCallPhases] = {};
    // Most recently used first; at most kShotPlans entries.
    static constexpr size_t kShotPlans = 4;
    std::vector<std::shared_ptr<ShotPlan>> plans_;
    // Used under dev_->mu; released (on the device's stream) before dev_.
    std::unique_ptr<SamplingWorkspace> ws_;
    void set_phase(int i, double v) {
        std::lock_guard<std::mutex> lk(mu_);
        phases_[i] = v;
    }
    uint64_t next_seed();
    ShotOutput run_shots(const std::vector<Operation>& ops, uint64_t n, uint64_t ncb, uint64_t shots, uint64_t seed,
                         bool profile, ShotPlan* plan = nullptr);
};

// Writes dqsim_profiles/statevector_shots_profile_<unix_ns>.json
// (src/profiling.rs:8-18); throws Error(kRuntimeError) on failure.
void write_shots_profile(const ShotOutput& out, double preprocessing, double fusion, double shots_total,
                         double total, uint64_t shots);

// Parse + validate + compile with no device work (host logic only).
std::vector<Operation> compile_json(const char* json, size_t len, uint64_t* n, uint64_t* ncb);

}  // namespace dq

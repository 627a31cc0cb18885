// Host-callable launchers of the per-gate statevector kernels (kernels.cu).
//
// Amplitudes are interleaved complex (c128: double2, c64: float2), little
// endian in the qubit index (qubit 0 is the least significant bit).  A batch
// holds W independent states of 2^n amplitudes back to back; every launcher
// covers the whole batch in one launch.  Classical bits are packed LSB-first,
// `cwords` 64-bit words per state, and stay on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.cuh"

namespace dq {
namespace k {

struct Batch {
    cudaStream_t stream = nullptr;
    bool c64 = false;
    void* amps = nullptr;
    int n = 0;
    uint64_t W = 1;
    uint64_t* cbits = nullptr;  // W * cwords words
    int cwords = 1;
    // Per-state measurement bookkeeping (device arrays of length W).
    uint64_t* rng_seed = nullptr;  // seed + shot of each state's ChaCha8 stream
    uint64_t* draws = nullptr;     // draws consumed so far
    int* outcome = nullptr;        // last outcome, -1 when the op was skipped
    double* scale = nullptr;       // 1/sqrt(p) of the last outcome
    double* partial = nullptr;     // W * kMaxChunks * 2 branch sums
    int* err = nullptr;            // set to 1 on a nonfinite or zero norm
};

constexpr int kMaxChunks = 1024;

struct Ctl {
    int qubit;
    bool value;
};

// (a, b) <- (u00 a + u01 b, u10 a + u11 b) on every (i, i + 2^t) pair whose
// controls hold; is_x swaps the pair instead (src/engine.rs:113-155).
void gate1q(const Batch& b, int target, const std::vector<Ctl>& controls, const double2 u[4], bool is_x,
            const dev::CondList& cond);

// Exchange amplitudes that differ in bits a, b (01 <-> 10) under controls (engine.rs:184-241).
void swap(const Batch& b, int qa, int qb, const std::vector<Ctl>& controls, const dev::CondList& cond);

// amp[i] *= diag[j(i)], qubits[0] the MSB of j (engine.rs:158-181).  Entries equal
// to exactly 1 are skipped when that leaves at most half of the table.
void diagonal(const Batch& b, const std::vector<int>& qubits, const std::vector<double2>& diag,
              const dev::CondList& cond);

// Dense 2^k x 2^k gate, k <= 5, row-major matrix already on the device (engine.rs:254-348).
void dense(const Batch& b, const std::vector<int>& qubits, const double2* dmatrix, const dev::CondList& cond);

// Measure (or reset) one qubit in every state whose condition holds: branch
// sums, a ChaCha8 draw per state, collapse (engine.rs:367-426).  cbit < 0: no write.
void measure(const Batch& b, int qubit, int64_t cbit, bool reset, const dev::CondList& cond);

// Measure one qubit of one state with a draw the caller supplies (uniform in
// [0, 1)): branch sums, outcome = draw < p1 / (p0 + p1), collapse; the outcome
// is returned to the host (the stream is synchronised).  engine.rs:367-426.
void measure_draw(const Batch& b, int qubit, double draw, int* outcome);
// out[i * 2^nl + j] = left[j] * right[i] (the merged block of two blocks).
void kron(cudaStream_t s, bool c64, const void* left, int nl, const void* right, int nr, void* out);

// Set each state to |0...0>.
void init_basis(const Batch& b);
// Copy one state into all W states of the batch.
void broadcast(const Batch& b, const void* src);

// |a_i|^2 into out (2^n doubles) for state 0.
void norm2(const Batch& b, double* out);
// Marginal probabilities over `qubits` (qubits[0] MSB) for state 0, 2^k doubles.
void marginal(const Batch& b, const std::vector<int>& qubits, double* out);
// In-place inclusive FP64 scan; `tmp` needs scan_tmp_size(len) doubles.
size_t scan_tmp_size(uint64_t len);
// Kernel launches scan (and scan_probs) makes for `len` entries.
int scan_launches(uint64_t len);
void scan(cudaStream_t s, double* x, uint64_t len, double* tmp);
// cdf[i] = cdf[i] / total (clamped to 1 when clamp), cdf[len-1] = 1.
void cdf_normalize(cudaStream_t s, double* cdf, uint64_t len, double total, bool clamp);
// Same with the total taken from cdf[len-1] on the device (copied to `scalar`
// first); sets *err when the total is not finite and positive.
void cdf_normalize_device(cudaStream_t s, double* cdf, uint64_t len, double* scalar, int* err, bool clamp);
// out[t] = min(partition_point(cdf, draw_t), len-1); per_shot_seed: draw_t is the
// first draw of seed+t, otherwise draw t of the stream `seed`.
void sample(cudaStream_t s, const double* cdf, uint64_t len, uint64_t seed, uint64_t shots, bool per_shot_seed,
            uint64_t* out);
// The same over unnormalised running sums: every probe normalises the entry it
// reads exactly as cdf_normalize would have (by *total_dev when given, else by
// total_host), so no normalising pass over the table is needed.  With `tiles`
// the sums are in two levels (scan_local): entry i is sums[i] plus
// tiles[i / 2048 - 1], the addition scan would have stored.
void sample_sums(cudaStream_t s, const double* sums, const double* tiles, uint64_t len, const double* total_dev,
                 double total_host, bool clamp, uint64_t seed, uint64_t shots, bool per_shot_seed, uint64_t* out);
// Inclusive running sums of state 0's squared magnitudes (in index order, the
// same values as norm2 then scan) into x; `tmp` needs scan_tmp_size(2^n)
// doubles.  add_tiles = false leaves them in two levels (see scan_local).
void scan_probs(const Batch& b, double* x, double* tmp, bool add_tiles = true);
// scan without its last pass: x holds sums within 2048-entry tiles and tmp[0..)
// the inclusive sums of whole tiles (entry i of the full scan is x[i] +
// tmp[i / 2048 - 1] for i >= 2048).
void scan_local(cudaStream_t s, double* x, uint64_t len, double* tmp);
uint64_t scan_tile_of(uint64_t i);
// *scalar = entry len-1 of the (two-level when tiles) sums; *err = 1 when it is
// not finite and positive.
void take_total(cudaStream_t s, const double* cdf, uint64_t len, const double* tiles, double* scalar, int* err);
// Partial sums of conj(a_i) * other_i (other is c128 on the device); returns block count.
int dot_partials(const Batch& b, const double2* other, double2* partial);
constexpr int kDotBlocks = 1184;
// c64 -> c128 widening copy of state 0.
void widen(const Batch& b, double2* out);
// out[j] = amplitude idx[j] of state 0 (device index list), widened to c128.
void gather(const Batch& b, const uint64_t* idx, uint64_t count, double2* out);
// Partial sums of (-1)^popcount((i^x)&z) conj(a_i) a_(i^x) for state 0; returns block count.
int pauli_partials(const Batch& b, uint64_t x, uint64_t z, double2* partial);
// Per-block partials of <a|b> and max |a_i - b_i| for two states of `len`
// amplitudes, each c128 or c64; partial holds kDotBlocks * 3 doubles.
// Per-block partials (kDotBlocks x 5): Re and Im of <a|b>, max |a_i - b_i|,
// <a|a> and <b|b>.
void compare(cudaStream_t s, const void* a, bool a64, const void* b, bool b64, uint64_t len, double* partial);

}  // namespace k
}  // namespace dq

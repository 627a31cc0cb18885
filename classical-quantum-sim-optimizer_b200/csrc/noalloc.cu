// Measurement of states the caller already holds on the device, with no
// device allocation anywhere on the call path.
//
// Some callers cannot call cudaMalloc: hosts whose device memory is owned and
// budgeted by their own allocator and that forbid side allocations, and
// latency-bound loops that cannot pay for the device-wide synchronisation
// cudaMalloc/cudaFree may trigger.  dq_measure_noalloc serves them: the states
// (inputs and outputs) are the caller's device memory, and the only scratch the
// measurement needs -- per-state seeds, draw counters, outcomes, scales, branch
// partial sums and an error flag -- lives in one file-scope __device__ array of
// fixed size, which every GPU that loads this library holds until the process
// exits.
//
// Ordering: the call issues its work on the legacy default stream and returns
// only after that work has finished (the outcomes are read back into host
// memory).  The legacy default stream does not wait for streams created
// non-blocking, so work that writes the states on such a stream (or on any
// stream of a per-thread-default-stream build) must be synchronised before the
// call.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dqsim_sv.h"
#include "common.hpp"
#include "kernels.hpp"

namespace dq {
namespace {

// Fixed scratch capacity.  Shared by every call on a device: calls whose work
// overlaps on the GPU (from several host threads or streams) race on it.
constexpr size_t kNoAllocScratchBytes = 256 * 1024;
static __device__ __align__(256) unsigned char g_measure_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Host code may not use g_measure_scratch as a device address: the name is a
// host-side stand-in.  The device address is looked up once per device, with
// that device current, on the first call made on it.
void* scratch_address(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (device < 0 || device >= kMaxDevices) fail(kValueError, "CUDA device ordinal out of range");
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_measure_scratch);
        if (e != cudaSuccess || !p)
            fail(kCudaError, std::string("cudaGetSymbolAddress(measurement scratch): ") + cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

// Measures `qubit` in each of num_states states of 2^num_qubits amplitudes
// held back to back at `states` (caller's device memory), drawing from the
// ChaCha8 stream seeds[i] at draw draw_index[i]; collapses (or resets) in
// place and writes each outcome to outcomes[i] (host memory).  A state whose
// norm is zero or not finite is left as it was with outcomes[i] = -1, and the
// call then fails with RuntimeError; every other state of the call has been
// measured and collapsed all the same, and its outcome is in outcomes[].
void measure_noalloc(void* states, int precision, uint64_t num_states, uint64_t num_qubits, uint64_t qubit, int reset,
                     const uint64_t* seeds, const uint64_t* draw_index, int* outcomes) {
    if (!states || !seeds || !draw_index || !outcomes) fail(kValueError, "null pointer argument");
    if (precision != DQ_COMPLEX128 && precision != DQ_COMPLEX64)
        fail(kValueError, "precision must be DQ_COMPLEX128 or DQ_COMPLEX64");
    if (num_states == 0) fail(kValueError, "num_states must be positive");
    if (num_qubits == 0 || num_qubits > 40) fail(kValueError, "num_qubits must be between 1 and 40");
    if (qubit >= num_qubits) fail(kValueError, "qubit is out of range");
    // Scratch layout: error flag | seeds | draws | outcomes | scales | partial sums.
    const uint64_t W = num_states;
    const int pbits = int(std::max<int64_t>(0, std::min<int64_t>(10, int64_t(num_qubits) - 12)));
    const uint64_t P = uint64_t(1) << pbits;
    if (W > kNoAllocScratchBytes / 8) fail(kValueError, "num_states exceeds the measurement scratch");
    const size_t o_err = 0, o_seed = 256, o_draw = o_seed + align256(W * 8), o_out = o_draw + align256(W * 8),
                 o_scale = o_out + align256(W * 4), o_part = o_scale + align256(W * 8);
    const size_t need = o_part + align256(W * P * 16);
    if (need > kNoAllocScratchBytes)
        fail(kValueError, "measuring " + std::to_string(W) + " states of " + std::to_string(num_qubits) +
                              " qubits needs " + std::to_string(need) + " bytes of scratch; the fixed measurement "
                              "scratch holds " + std::to_string(kNoAllocScratchBytes) + " bytes (use fewer states per call)");
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, states) != cudaSuccess ||
        (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        fail(kValueError, "states must point to CUDA device memory");
    }
    const int device = attr.device;
    int current = 0;
    if (cudaGetDevice(&current) != cudaSuccess) fail(kCudaError, "cudaGetDevice failed");
    if (current != device && cudaSetDevice(device) != cudaSuccess) fail(kCudaError, "cudaSetDevice failed");
    struct Restore {
        int dev, cur;
        ~Restore() {
            if (dev != cur) cudaSetDevice(cur);
        }
    } restore{device, current};
    unsigned char* base = static_cast<unsigned char*>(scratch_address(device));
    cudaStream_t s = nullptr;  // legacy default stream
    // The array keeps the previous call's contents: the error flag must start at zero.
    if (cudaMemsetAsync(base + o_err, 0, 16, s) != cudaSuccess ||
        cudaMemcpyAsync(base + o_seed, seeds, W * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(base + o_draw, draw_index, W * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
        fail(kCudaError, std::string("scratch upload: ") + cudaGetErrorString(cudaGetLastError()));
    k::Batch b;
    b.stream = s;
    b.c64 = precision == DQ_COMPLEX64;
    b.amps = states;
    b.n = int(num_qubits);
    b.W = W;
    b.cbits = reinterpret_cast<uint64_t*>(base + o_err);  // never written: no classical bit (cbit < 0)
    b.cwords = 1;
    b.rng_seed = reinterpret_cast<uint64_t*>(base + o_seed);
    b.draws = reinterpret_cast<uint64_t*>(base + o_draw);
    b.outcome = reinterpret_cast<int*>(base + o_out);
    b.scale = reinterpret_cast<double*>(base + o_scale);
    b.partial = reinterpret_cast<double*>(base + o_part);
    b.err = reinterpret_cast<int*>(base + o_err + 8);
    dev::CondList none{};
    k::measure(b, int(qubit), -1, reset != 0, none);
    int flag = 0;
    if (cudaMemcpy(outcomes, base + o_out, W * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&flag, base + o_err + 8, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        fail(kCudaError, std::string("reading outcomes: ") + cudaGetErrorString(cudaGetLastError()));
    if (flag) fail(kRuntimeError, "Cannot measure a state with nonfinite or zero norm");
}

}  // namespace dq

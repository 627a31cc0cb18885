// Dense blocks of the P-block backend on the device.
//
// The reference's P-block backend (src/distributed/pblock/model.rs) keeps the
// state as independent dense blocks of qubits and runs every gate, merge and
// measurement on one block with the dense kernels of src/engine.rs:
// apply_one_qubit / apply_x (model.rs:318-325), apply_swap (:370),
// apply_diagonal (:415), DenseLayout::apply (:429), measure_qubit (:484-486),
// the merge of two blocks into their product state (:199-248) and the running
// sums of each block's squared magnitudes it samples from (:583-608).  A
// BlockContext runs those operations on blocks the caller keeps in device
// memory (complex128 or complex64, little-endian in the block's local qubits),
// in order on its own stream, with the statevector engine's kernels; the block
// bookkeeping (which qubits a block holds, when to merge or split) stays with
// the caller, as it does in model.rs.
#include "blocks.hpp"

#include <algorithm>
#include <string>

namespace dq {

BlockContext::BlockContext(int device, bool c64) : device_(device), c64_(c64) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        fail(kValueError, "CUDA device ordinal out of range");
    }
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    outcome_.alloc(16, "block measurement outcome");
    scale_.alloc(16, "block measurement scale");
    partial_.alloc(size_t(k::kMaxChunks) * 2 * 8, "block branch sums");
    cbits_.alloc(16, "block classical bits");
    err_.alloc(16, "block error flag");
}

BlockContext::~BlockContext() {
    if (stream_) {
        cudaSetDevice(device_);
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
}

k::Batch BlockContext::batch(void* state, uint64_t n) {
    if (!state) fail(kValueError, "null block state");
    if (n == 0 || n > 40) fail(kValueError, "a block holds 1 to 40 qubits");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    k::Batch b;
    b.stream = stream_;
    b.c64 = c64_;
    b.amps = state;
    b.n = int(n);
    b.W = 1;
    b.cbits = cbits_.as<uint64_t>();
    b.cwords = 1;
    b.outcome = outcome_.as<int>();
    b.scale = scale_.as<double>();
    b.partial = partial_.as<double>();
    b.err = err_.as<int>();
    return b;
}

namespace {

std::vector<k::Ctl> controls_of(uint64_t n, uint64_t target, const uint64_t* qubits, const uint8_t* values, size_t count,
                                const std::vector<uint64_t>& also) {
    std::vector<k::Ctl> cs;
    std::vector<uint64_t> used(also);
    used.push_back(target);
    for (size_t i = 0; i < count; i++) {
        if (qubits[i] >= n || std::find(used.begin(), used.end(), qubits[i]) != used.end())
            fail(kValueError, "block control qubits must be distinct block qubits other than the targets");
        used.push_back(qubits[i]);
        cs.push_back({int(qubits[i]), values[i] != 0});
    }
    return cs;
}

std::vector<int> qubit_list(uint64_t n, const uint64_t* qubits, size_t k, size_t max_k) {
    if (k == 0 || k > max_k) fail(kValueError, "block gates take 1 to " + std::to_string(max_k) + " qubits");
    std::vector<int> q;
    for (size_t i = 0; i < k; i++) {
        if (qubits[i] >= n || std::find(q.begin(), q.end(), int(qubits[i])) != q.end())
            fail(kValueError, "block gate qubits must be distinct block qubits");
        q.push_back(int(qubits[i]));
    }
    return q;
}

}  // namespace

void BlockContext::apply_one_qubit(void* state, uint64_t n, uint64_t target, const double* m, const uint64_t* cq,
                                   const uint8_t* cv, size_t nc, bool is_x) {
    k::Batch b = batch(state, n);
    if (target >= n) fail(kValueError, "target is not a block qubit");
    if (nc && (!cq || !cv)) fail(kValueError, "null control list");
    std::vector<k::Ctl> cs = controls_of(n, target, cq, cv, nc, {});
    double2 u[4] = {};
    if (!is_x) {
        if (!m) fail(kValueError, "null matrix");
        for (int i = 0; i < 4; i++) u[i] = make_double2(m[2 * i], m[2 * i + 1]);
    }
    k::gate1q(b, int(target), cs, u, is_x, dev::CondList{});
}

void BlockContext::apply_swap(void* state, uint64_t n, uint64_t a, uint64_t bq, const uint64_t* cq, const uint8_t* cv,
                              size_t nc) {
    k::Batch b = batch(state, n);
    if (a >= n || bq >= n || a == bq) fail(kValueError, "swap qubits must be two distinct block qubits");
    if (nc && (!cq || !cv)) fail(kValueError, "null control list");
    std::vector<k::Ctl> cs = controls_of(n, a, cq, cv, nc, {bq});
    k::swap(b, int(a), int(bq), cs, dev::CondList{});
}

void BlockContext::apply_diagonal(void* state, uint64_t n, const uint64_t* qubits, size_t kq, const double* diag) {
    k::Batch b = batch(state, n);
    if (!qubits || !diag) fail(kValueError, "null diagonal argument");
    std::vector<int> q = qubit_list(n, qubits, kq, 5);
    std::vector<double2> d(size_t(1) << kq);
    for (size_t i = 0; i < d.size(); i++) d[i] = make_double2(diag[2 * i], diag[2 * i + 1]);
    k::diagonal(b, q, d, dev::CondList{});
}

void BlockContext::apply_dense(void* state, uint64_t n, const uint64_t* qubits, size_t kq, const double* matrix) {
    k::Batch b = batch(state, n);
    if (!qubits || !matrix) fail(kValueError, "null dense argument");
    std::vector<int> q = qubit_list(n, qubits, kq, 5);
    const size_t entries = size_t(1) << (2 * kq);
    // The matrix buffer is reused by the next call: wait for the previous gate to read it.
    cuda_check(cudaStreamSynchronize(stream_), "stream synchronize");
    mat_.ensure(entries * sizeof(double2), "block gate matrix");
    cuda_check(cudaMemcpyAsync(mat_.p, matrix, entries * sizeof(double2), cudaMemcpyHostToDevice, stream_),
               "upload block gate matrix");
    k::dense(b, q, mat_.as<double2>(), dev::CondList{});
}

int BlockContext::measure(void* state, uint64_t n, uint64_t qubit, double draw) {
    k::Batch b = batch(state, n);
    if (qubit >= n) fail(kValueError, "qubit is not a block qubit");
    if (!(draw >= 0.0 && draw < 1.0)) fail(kValueError, "the draw must lie in [0, 1)");
    int outcome = 0;
    k::measure_draw(b, int(qubit), draw, &outcome);
    return outcome;
}

void BlockContext::merge(const void* left, uint64_t nl, const void* right, uint64_t nr, void* out) {
    if (!left || !right || !out) fail(kValueError, "null block state");
    if (nl == 0 || nr == 0 || nl + nr > 40) fail(kValueError, "a merged block holds 2 to 40 qubits");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    k::kron(stream_, c64_, left, int(nl), right, int(nr), out);
}

void BlockContext::probabilities(const void* state, uint64_t n, const uint64_t* qubits, size_t kq, double* out) {
    k::Batch b = batch(const_cast<void*>(state), n);
    if (!out) fail(kValueError, "null output");
    if (kq == 0) {
        k::norm2(b, out);
        return;
    }
    if (!qubits) fail(kValueError, "null qubit list");
    std::vector<int> q = qubit_list(n, qubits, kq, 40);
    k::marginal(b, q, out);
}

void BlockContext::running_sums(const void* state, uint64_t n, double* out) {
    k::Batch b = batch(const_cast<void*>(state), n);
    if (!out) fail(kValueError, "null output");
    // The scratch is reused by the next call: wait for the previous one to finish with it.
    cuda_check(cudaStreamSynchronize(stream_), "stream synchronize");
    tmp_.ensure(k::scan_tmp_size(uint64_t(1) << n) * 8, "block scan scratch");
    k::scan_probs(b, out, tmp_.as<double>(), true);
}

void BlockContext::sync() {
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaStreamSynchronize(stream_), "stream synchronize");
}

}  // namespace dq

#include "cost.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "common.hpp"
#include "engine.hpp"

namespace dq {
namespace {

constexpr int F = kMlpF, H = kMlpH, B = kMlpB;
constexpr int oW1 = 0, ob1 = H * F, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + H;
constexpr int kTrainThreads = 256;
// Extra slots after the parameters: target mean and standard deviation.
constexpr int kStored = kMlpParams + 2;

struct TrainSmem {
    static constexpr size_t floats = size_t(B) * F + 3 * size_t(B) * H + 2 * B + kMlpParams;
};

__global__ void __launch_bounds__(kTrainThreads) k_mlp_train(float* __restrict__ P, float* __restrict__ Am,
                                                            float* __restrict__ Av, const float* __restrict__ X,
                                                            const float* __restrict__ Y, const int* __restrict__ perm,
                                                            int N, int steps, int t0, float lr,
                                                            float* __restrict__ loss_out, float* __restrict__ grad_out,
                                                            int nbatch) {
    extern __shared__ float sm[];
    float* x = sm;
    float* a1 = x + B * F;
    float* a2 = a1 + B * H;
    float* d = a2 + B * H;
    float* dy = d + B * H;
    float* err = dy + B;
    float* g = err + B;
    const int tid = threadIdx.x, nt = blockDim.x;
    float loss_sum = 0.f;
    for (int s = 0; s < steps; s++) {
        const int rows = nbatch;  // rows of this batch
        for (int o = tid; o < B * F; o += nt) {
            int r = o / F;
            x[o] = r < rows ? X[size_t(perm[(size_t(s) * B + r) % N]) * F + (o % F)] : 0.f;
        }
        __syncthreads();
        for (int o = tid; o < B * H; o += nt) {
            int r = o / H, h = o % H;
            float z = P[ob1 + h];
            for (int f = 0; f < F; f++) z += P[oW1 + h * F + f] * x[r * F + f];
            a1[o] = z > 0.f ? z : 0.f;
        }
        __syncthreads();
        for (int o = tid; o < B * H; o += nt) {
            int r = o / H, h = o % H;
            float z = P[ob2 + h];
            for (int k = 0; k < H; k++) z += P[oW2 + h * H + k] * a1[r * H + k];
            a2[o] = z > 0.f ? z : 0.f;
        }
        __syncthreads();
        for (int r = tid; r < B; r += nt) {
            float yp = P[ob3];
            for (int h = 0; h < H; h++) yp += P[oW3 + h] * a2[r * H + h];
            float diff = r < rows ? yp - Y[perm[(size_t(s) * B + r) % N]] : 0.f;
            err[r] = diff * diff;
            dy[r] = 2.f * diff / float(rows);
        }
        __syncthreads();
        if (tid == 0) {
            float l = 0.f;
            for (int r = 0; r < rows; r++) l += err[r];
            loss_sum += l / float(rows);
        }
        for (int h = tid; h < H; h += nt) {
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += dy[r] * a2[r * H + h];
            g[oW3 + h] = acc;
        }
        if (tid == 0) {
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += dy[r];
            g[ob3] = acc;
        }
        for (int o = tid; o < B * H; o += nt) {
            int r = o / H, h = o % H;
            d[o] = a2[o] > 0.f ? dy[r] * P[oW3 + h] : 0.f;  // dZ2
        }
        __syncthreads();
        for (int o = tid; o < H * H; o += nt) {
            int h = o / H, k = o % H;
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += d[r * H + h] * a1[r * H + k];
            g[oW2 + o] = acc;
        }
        for (int h = tid; h < H; h += nt) {
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += d[r * H + h];
            g[ob2 + h] = acc;
        }
        // dZ1 overwrites a2 (no longer needed)
        for (int o = tid; o < B * H; o += nt) {
            int r = o / H, k = o % H;
            float acc = 0.f;
            for (int h = 0; h < H; h++) acc += d[r * H + h] * P[oW2 + h * H + k];
            a2[o] = a1[o] > 0.f ? acc : 0.f;
        }
        __syncthreads();
        for (int o = tid; o < H * F; o += nt) {
            int k = o / F, f = o % F;
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += a2[r * H + k] * x[r * F + f];
            g[oW1 + o] = acc;
        }
        for (int k = tid; k < H; k += nt) {
            float acc = 0.f;
            for (int r = 0; r < B; r++) acc += a2[r * H + k];
            g[ob1 + k] = acc;
        }
        __syncthreads();
        if (grad_out) {
            for (int p = tid; p < kMlpParams; p += nt) grad_out[p] = g[p];
            return;
        }
        const float b1m = 0.9f, b2v = 0.999f, eps = 1e-8f;
        const float t = float(t0 + s + 1);
        const float c1 = 1.f - powf(b1m, t), c2 = 1.f - powf(b2v, t);
        for (int p = tid; p < kMlpParams; p += nt) {
            float gp = g[p];
            float m = b1m * Am[p] + (1.f - b1m) * gp;
            float v = b2v * Av[p] + (1.f - b2v) * gp * gp;
            Am[p] = m;
            Av[p] = v;
            P[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
        }
        __syncthreads();
    }
    if (tid == 0 && loss_out) *loss_out = loss_sum / float(steps > 0 ? steps : 1);
}

__global__ void k_mlp_infer(const float* __restrict__ P, const float* __restrict__ X, int n, float* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x[F];
#pragma unroll
    for (int f = 0; f < F; f++) x[f] = X[size_t(i) * F + f];
    float h1[H];
#pragma unroll 4
    for (int h = 0; h < H; h++) {
        float z = P[ob1 + h];
#pragma unroll
        for (int f = 0; f < F; f++) z += P[oW1 + h * F + f] * x[f];
        h1[h] = z > 0.f ? z : 0.f;
    }
    float y = P[ob3];
    for (int h = 0; h < H; h++) {
        float z = P[ob2 + h];
#pragma unroll
        for (int k = 0; k < H; k++) z += P[oW2 + h * H + k] * h1[k];
        y += P[oW3 + h] * (z > 0.f ? z : 0.f);
    }
    out[i] = y;
}

size_t train_smem() { return TrainSmem::floats * sizeof(float); }

}  // namespace

void tile_op_features(const TileOp& op, int m, bool c64, float* out) {
    for (int i = 0; i < F; i++) out[i] = 0.f;
    out[op.type] = 1.f;  // 0..5
    int lo = 31, hi = 0, count = 0;
    auto see = [&](int p) {
        lo = std::min(lo, p);
        hi = std::max(hi, p);
        count++;
    };
    int items_log = m;
    switch (op.type) {
        case TileOp::kDiagFull:
            for (int b = 0; b < op.k; b++) see(op.q[b]);
            items_log = m;
            break;
        case TileOp::kDense:
            for (int b = 0; b < op.k; b++) see(op.q[b]);
            items_log = m - op.k;
            break;
        default:
            for (int b = 0; b < op.nins; b++) see(op.ins[b]);
            items_log = m - op.nins;
            break;
    }
    if (count == 0) lo = hi = 0;
    const int k = op.type == TileOp::kDense || op.type == TileOp::kDiagFull ? op.k : op.nins;
    out[6] = float(k) / 5.f;
    out[7] = float(op.nins) / 7.f;
    out[8] = float(std::max(1, op.ngates)) / 16.f;
    out[9] = float(lo) / 14.f;
    out[10] = float(hi) / 14.f;
    out[11] = lo < 3 ? 1.f : 0.f;
    out[12] = float(items_log) / 14.f;
    out[13] = float(m) / 14.f;
    out[14] = c64 ? 1.f : 0.f;
    out[15] = float(count) / 5.f;
}

void fused_block_features(int gates, uint32_t local_mask, int nblocks, float* out) {
    for (int i = 0; i < F; i++) out[i] = 0.f;
    int lo = 31, hi = 0;
    for (int b = 0; b < 32; b++)
        if ((local_mask >> b) & 1u) {
            lo = std::min(lo, b);
            hi = std::max(hi, b);
        }
    if (local_mask == 0) lo = hi = 0;
    out[6] = 1.f;  // width 5: only tensor-core blocks have it
    out[7] = 1.f / float(std::max(1, nblocks));
    out[8] = float(std::max(1, gates)) / 16.f;
    out[9] = float(lo) / 14.f;
    out[10] = float(hi) / 14.f;
    out[11] = lo < 3 ? 1.f : 0.f;
    out[12] = float(kFusedM - 5) / 14.f;
    out[13] = float(kFusedM) / 14.f;
    out[14] = 1.f;
    out[15] = 1.f;
}

void fused_pass_features(int n, uint64_t states, const std::vector<int>& tile_qubits, int nblocks, int gates,
                         float* out) {
    for (int i = 0; i < F; i++) out[i] = 0.f;
    uint64_t T = 0;
    for (int q : tile_qubits) T |= uint64_t(1) << q;
    const int nb = std::max(1, nblocks);
    out[0] = float(n) / 32.f;
    out[1] = float(nblocks) / 8.f;
    out[2] = 1.f / float(nb);
    // Tile qubits by position (stride 8 B << q in the state), in bins of four
    // from qubit 2 (qubits 0 and 1 are in every fused tile).
    for (int q : tile_qubits)
        if (q >= kFusedPinned) out[3 + std::min(7, (q - kFusedPinned) / 4)] += 0.25f;
    int top = 0;
    for (int q : tile_qubits) top += q >= n - 3 ? 1 : 0;
    out[11] = float(top) / 3.f;
    // The ingredients of the hand rule: tile qubits lengthening the runs that
    // the ~2^9 tiles in flight read together, and where those runs end.
    int run_bits = 0, outside = 0, c = n;
    for (int q = 0; q < n; q++) {
        if ((T >> q) & 1) {
            run_bits += q >= kFusedPinned ? 1 : 0;
        } else if (++outside > 9) {
            c = q;
            break;
        }
    }
    out[12] = float(run_bits) / 8.f;
    out[13] = float(c) / 32.f;
    const FusedTma tma = fused_tma_plan(tile_qubits, n, states);
    out[14] = tma.ok ? std::log2(float(tma.copies)) / 4.f : 1.25f;  // per-thread loads without TMA
    out[15] = float(gates) / (16.f * float(nb));
}

CostModel::CostModel(int device, uint64_t seed, int kind) : device_(device), kind_(kind) {
    if (kind != kCostTileOps && kind != kCostFusedPasses) fail(kValueError, "unknown cost model kind");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaMalloc(&params_, sizeof(float) * (3 * size_t(kStored))), "cost model parameters");
    std::vector<float> p(3 * size_t(kStored), 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int i = 0; i < H * F; i++) p[oW1 + i] = nd(rng) * std::sqrt(2.f / F);
    for (int i = 0; i < H * H; i++) p[oW2 + i] = nd(rng) * std::sqrt(2.f / H);
    for (int i = 0; i < H; i++) p[oW3 + i] = nd(rng) * std::sqrt(1.f / H);
    p[kMlpParams] = 0.f;      // target mean
    p[kMlpParams + 1] = 1.f;  // target std
    cuda_check(cudaMemcpy(params_, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(train_smem())),
               "smem attribute");
}

CostModel::~CostModel() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (params_) cudaFree(params_);
    if (stream_) cudaStreamDestroy(stream_);
}

void CostModel::add_samples(const float* X, const float* y, size_t n) {
    std::lock_guard<std::mutex> lk(mu_);
    X_.insert(X_.end(), X, X + n * F);
    y_.insert(y_.end(), y, y + n);
}

double CostModel::train(int epochs, float lr) {
    std::lock_guard<std::mutex> lk(mu_);
    const size_t N = y_.size();
    if (N < size_t(B)) fail(kValueError, "the cost model needs at least 128 samples to train");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    // Targets normalised to zero mean / unit variance; the statistics ride with the weights.
    double mu = 0, var = 0;
    for (float v : y_) mu += v;
    mu /= double(N);
    for (float v : y_) var += (v - mu) * (v - mu);
    const double sd = std::max(1e-6, std::sqrt(var / double(N)));
    std::vector<float> yn(N);
    for (size_t i = 0; i < N; i++) yn[i] = float((y_[i] - mu) / sd);
    float stats[2] = {float(mu), float(sd)};
    float* P = static_cast<float*>(params_);
    cuda_check(cudaMemcpyAsync(P + kMlpParams, stats, 8, cudaMemcpyHostToDevice, stream_), "upload");
    DevMem dX, dY, dperm, dloss;
    dX.alloc(X_.size() * 4, "training features");
    dY.alloc(N * 4, "training targets");
    dperm.alloc(N * 4, "permutation");
    dloss.alloc(16, "loss");
    cuda_check(cudaMemcpyAsync(dX.p, X_.data(), X_.size() * 4, cudaMemcpyHostToDevice, stream_), "upload");
    cuda_check(cudaMemcpyAsync(dY.p, yn.data(), N * 4, cudaMemcpyHostToDevice, stream_), "upload");
    // Fresh Adam state for each training call.
    cuda_check(cudaMemsetAsync(P + kStored, 0, sizeof(float) * 2 * kStored, stream_), "clear adam");
    std::vector<int> perm(N);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(12345);
    const int steps = int((N + B - 1) / B);
    float loss = 0.f;
    for (int e = 0; e < epochs; e++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        cuda_check(cudaMemcpyAsync(dperm.p, perm.data(), N * 4, cudaMemcpyHostToDevice, stream_), "upload");
        k_mlp_train<<<1, kTrainThreads, train_smem(), stream_>>>(P, P + kStored, P + 2 * kStored, dX.as<float>(),
                                                                 dY.as<float>(), dperm.as<int>(), int(N), steps,
                                                                 e * steps, lr, dloss.as<float>(), nullptr, B);
        cuda_check(cudaGetLastError(), "mlp train launch");
        cuda_check(cudaMemcpyAsync(&loss, dloss.p, 4, cudaMemcpyDeviceToHost, stream_), "read loss");
        cuda_check(cudaStreamSynchronize(stream_), "sync");
    }
    trained_ = true;
    return double(loss);
}

void CostModel::gradients(const float* X, const float* y, size_t n, float* grads) const {
    std::lock_guard<std::mutex> lk(mu_);
    if (n == 0 || n > size_t(B)) fail(kValueError, "gradient batches hold 1..128 samples");
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    DevMem dX, dY, dperm, dg;
    dX.alloc(n * F * 4, "features");
    dY.alloc(n * 4, "targets");
    dperm.alloc(n * 4, "permutation");
    dg.alloc(kMlpParams * 4, "gradients");
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    cuda_check(cudaMemcpyAsync(dX.p, X, n * F * 4, cudaMemcpyHostToDevice, stream_), "upload");
    cuda_check(cudaMemcpyAsync(dY.p, y, n * 4, cudaMemcpyHostToDevice, stream_), "upload");
    cuda_check(cudaMemcpyAsync(dperm.p, perm.data(), n * 4, cudaMemcpyHostToDevice, stream_), "upload");
    float* P = static_cast<float*>(params_);
    k_mlp_train<<<1, kTrainThreads, train_smem(), stream_>>>(P, P + kStored, P + 2 * kStored, dX.as<float>(),
                                                             dY.as<float>(), dperm.as<int>(), int(n), 1, 0, 0.f,
                                                             nullptr, dg.as<float>(), int(n));
    cuda_check(cudaGetLastError(), "mlp gradient launch");
    cuda_check(cudaMemcpyAsync(grads, dg.p, kMlpParams * 4, cudaMemcpyDeviceToHost, stream_), "read gradients");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
}

void CostModel::predict(const float* X, size_t n, float* out) const {
    std::lock_guard<std::mutex> lk(mu_);
    if (n == 0) return;
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    DevMem dX, dO;
    dX.alloc(n * F * 4, "features");
    dO.alloc(n * 4, "predictions");
    cuda_check(cudaMemcpyAsync(dX.p, X, n * F * 4, cudaMemcpyHostToDevice, stream_), "upload");
    k_mlp_infer<<<unsigned((n + 127) / 128), 128, 0, stream_>>>(static_cast<const float*>(params_), dX.as<float>(),
                                                                int(n), dO.as<float>());
    cuda_check(cudaGetLastError(), "mlp infer launch");
    cuda_check(cudaMemcpyAsync(out, dO.p, n * 4, cudaMemcpyDeviceToHost, stream_), "read predictions");
    float stats[2];
    cuda_check(cudaMemcpyAsync(stats, static_cast<float*>(params_) + kMlpParams, 8, cudaMemcpyDeviceToHost, stream_),
               "read stats");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    for (size_t i = 0; i < n; i++) out[i] = stats[0] + stats[1] * out[i];
}

void CostModel::get_params(float* out) const {
    std::lock_guard<std::mutex> lk(mu_);
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaMemcpy(out, params_, sizeof(float) * kStored, cudaMemcpyDeviceToHost), "read parameters");
}

void CostModel::set_params(const float* in) {
    std::lock_guard<std::mutex> lk(mu_);
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    cuda_check(cudaMemcpy(params_, in, sizeof(float) * kStored, cudaMemcpyHostToDevice), "write parameters");
    trained_ = true;
}

double CostModel::predict_ops(const std::vector<TileOp>& ops, int m, bool c64) const {
    if (ops.empty()) return 0.0;
    std::vector<float> X(ops.size() * F), y(ops.size());
    for (size_t i = 0; i < ops.size(); i++) tile_op_features(ops[i], m, c64, X.data() + i * F);
    predict(X.data(), ops.size(), y.data());
    double total = 0;
    for (float v : y) total += std::exp(double(v));
    return total;
}

double CostModel::predict_fused(const FusedPass& p) const {
    const size_t nb = p.block_gates.size();
    if (nb == 0) return 0.0;
    std::vector<float> X(nb * F), y(nb);
    for (size_t i = 0; i < nb; i++) fused_block_features(p.block_gates[i], p.block_masks[i], int(nb), X.data() + i * F);
    predict(X.data(), nb, y.data());
    double total = 0;
    for (float v : y) total += std::exp(double(v));
    return total;
}

std::vector<double> CostModel::predict_passes_ms(const FusedPortfolio& pf, uint64_t states) const {
    const size_t np = pf.built.size();
    std::vector<double> ms(np, 0.0);
    if (np == 0) return ms;
    std::vector<float> X(np * F), y(np);
    for (size_t i = 0; i < np; i++) {
        const FusedPass& fp = pf.built[i].fp;
        int gates = 0;
        for (int g : fp.block_gates) gates += g;
        fused_pass_features(pf.n, states, fp.qubits, fp.nblocks, gates, X.data() + i * F);
    }
    predict(X.data(), np, y.data());
    const double tiles = double(states << (pf.n - kFusedM));
    for (size_t i = 0; i < np; i++) ms[i] = std::exp(double(y[i])) * tiles * 1e-6;  // ns per tile -> ms
    return ms;
}

std::vector<double> CostModel::predict_plans_ms(const FusedPortfolio& pf, uint64_t states) const {
    const std::vector<double> pass_ms = predict_passes_ms(pf, states);
    std::vector<double> plan_ms(pf.plans.size(), 0.0);
    for (size_t i = 0; i < pf.plans.size(); i++)
        for (size_t slot : pf.slots[i]) plan_ms[i] += pass_ms[slot];
    return plan_ms;
}

}  // namespace dq

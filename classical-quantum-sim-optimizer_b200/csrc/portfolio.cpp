// Candidate fused plans and single fused passes, timed on the device: the
// training data and the ground truth of the learned pass-cost model.
//
// fused_portfolio_json lists every candidate plan of a circuit's unitary
// prefix (one per spread cap), each distinct pass's features (the
// kCostFusedPasses model's inputs), the hand rule's cost of each plan and its
// choice, and optionally each pass's measured device time (k_fused on a
// complex64 state of the circuit's size) and a model's predictions.
// fused_random_passes_json builds seeded random passes (random tile qubits,
// random one- and two-qubit gates clustered into 1..10 blocks) and times them
// the same way.
#include "portfolio.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>

#include "cost.hpp"
#include "engine.hpp"

namespace dq {
namespace {

// Times single fused passes over one complex64 state of n qubits.
class PassTimer {
  public:
    PassTimer(Simulator& sim, int n) : dev_(sim.ensure_device()), n_(n) {
        std::lock_guard<std::mutex> lk(dev_->mu);
        dev_->activate();
        st_.allocate(n, 1, 0, true, dev_->stream);
        k::Batch b = st_.view(dev_->stream, 1);
        k::init_basis(b);
        cuda_check(cudaMemsetAsync(st_.err.p, 0, 16, dev_->stream), "clear error flag");
        tnorm_.alloc((size_t(1) << (n - kFusedM)) * 8, "fused tile norms");
        cuda_check(cudaEventCreate(&e0_), "cudaEventCreate");
        cuda_check(cudaEventCreate(&e1_), "cudaEventCreate");
    }
    ~PassTimer() {
        cudaEventDestroy(e0_);
        cudaEventDestroy(e1_);
    }
    // Device milliseconds of one launch of the pass (the faster of two, after one untimed).
    double time(const BuiltFusedPass& p) {
        std::lock_guard<std::mutex> lk(dev_->mu);
        dev_->activate();
        cudaStream_t s = dev_->stream;
        blocks_.ensure(p.blocks.size() * sizeof(FusedBlock), "fused block descriptors");
        upool_.ensure(p.upool.size() * sizeof(uint16_t), "fused block gate images");
        cuda_check(cudaMemcpyAsync(blocks_.p, p.blocks.data(), p.blocks.size() * sizeof(FusedBlock),
                                   cudaMemcpyHostToDevice, s),
                   "upload fused blocks");
        cuda_check(cudaMemcpyAsync(upool_.p, p.upool.data(), p.upool.size() * sizeof(uint16_t), cudaMemcpyHostToDevice,
                                   s),
                   "upload gate images");
        k::Batch b = st_.view(s, 1);
        double best = 1e30;
        for (int rep = 0; rep < 3; rep++) {
            cuda_check(cudaEventRecord(e0_, s), "cudaEventRecord");
            k::fused_pass(b, p.fp, blocks_.as<FusedBlock>(), upool_.as<uint16_t>(), st_.err.as<int>(), nullptr,
                          tnorm_.as<double>());
            cuda_check(cudaEventRecord(e1_, s), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(e1_), "cudaEventSynchronize");
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e0_, e1_), "cudaEventElapsedTime");
            if (rep > 0) best = std::min(best, double(ms));
        }
        int flag = 0;
        cuda_check(cudaMemcpy(&flag, st_.err.p, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
        if (flag == 3) fail(kRuntimeError, "a tensor-core pass gave up on a bounded wait");
        return best;
    }

  private:
    std::shared_ptr<Device> dev_;
    int n_;
    StateBatch st_;
    DevMem tnorm_, blocks_, upool_;
    cudaEvent_t e0_ = nullptr, e1_ = nullptr;
};

std::string num(double v) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.6g", v);
    return buf;
}

// One distinct pass as JSON: tile qubits, blocks, gates, features, and the
// measured / predicted milliseconds (negative when not asked for).
std::string pass_json(int n, const FusedPass& fp, double ms, double pred_ms) {
    int gates = 0;
    for (int g : fp.block_gates) gates += g;
    float f[kMlpF];
    fused_pass_features(n, 1, fp.qubits, fp.nblocks, gates, f);
    std::string s = "{\"qubits\": [";
    for (size_t i = 0; i < fp.qubits.size(); i++) s += (i ? ", " : "") + std::to_string(fp.qubits[i]);
    s += "], \"blocks\": " + std::to_string(fp.nblocks) + ", \"gates\": " + std::to_string(gates) + ", \"features\": [";
    for (int i = 0; i < kMlpF; i++) s += (i ? ", " : "") + num(f[i]);
    s += "], \"ms\": " + num(ms) + ", \"predicted_ms\": " + num(pred_ms) + "}";
    return s;
}

// A seeded random unitary 2x2 (U3 with uniform angles).
Mat2 random_u3(std::mt19937_64& rng) {
    std::uniform_real_distribution<double> u(0.0, 2.0 * M_PI);
    const double th = u(rng), ph = u(rng), la = u(rng);
    const double c = std::cos(th / 2), s = std::sin(th / 2);
    Mat2 m;
    m[0][0] = cplx(c, 0);
    m[0][1] = cplx(-std::cos(la) * s, -std::sin(la) * s);
    m[1][0] = cplx(std::cos(ph) * s, std::sin(ph) * s);
    m[1][1] = cplx(std::cos(ph + la) * c, std::sin(ph + la) * c);
    return m;
}

}  // namespace

std::string fused_portfolio_json(Simulator& sim, const char* json, size_t len, bool wide, bool measure,
                                 const CostModel* model) {
    uint64_t n = 0, ncb = 0;
    std::vector<Operation> ops = compile_json(json, len, &n, &ncb);
    size_t end = ops.size();
    for (size_t i = 0; i < ops.size(); i++)
        if (!ops[i].is_unitary()) {
            end = i;
            break;
        }
    if (n < uint64_t(kFusedM)) fail(kValueError, "fused passes need at least 12 qubits");
    if (n > 34) fail(kValueError, "fused portfolios are timed on states of at most 34 qubits");
    if (model && model->kind() != kCostFusedPasses) fail(kValueError, "the model does not price fused passes");
    FusedPortfolio pf = fused_portfolio(ops, 0, end, int(n), TilePlanOptions{}, fused_caps(int(n), wide));
    std::vector<double> ms(pf.built.size(), -1.0), pred(pf.built.size(), -1.0);
    if (measure) {
        PassTimer timer(sim, int(n));
        for (size_t i = 0; i < pf.built.size(); i++) ms[i] = timer.time(pf.built[i]);
    }
    if (model) pred = model->predict_passes_ms(pf, 1);
    std::string s = "{\"n\": " + std::to_string(n) + ", \"ops\": " + std::to_string(end) +
                    ", \"rule_choice\": " + std::to_string(pf.rule_choice) + ", \"plans\": [";
    for (size_t i = 0; i < pf.plans.size(); i++) {
        s += i ? ", {" : "{";
        s += "\"cap\": " + std::to_string(pf.caps[i]) + ", \"rule_cost\": " + num(pf.rule_cost[i]) + ", \"passes\": [";
        for (size_t k = 0; k < pf.slots[i].size(); k++) s += (k ? ", " : "") + std::to_string(pf.slots[i][k]);
        s += "]}";
    }
    s += "], \"passes\": [";
    for (size_t i = 0; i < pf.built.size(); i++) s += (i ? ", " : "") + pass_json(int(n), pf.built[i].fp, ms[i], pred[i]);
    return s + "]}";
}

std::string fused_random_passes_json(Simulator& sim, int n, uint64_t count, uint64_t seed, bool measure) {
    if (n < kFusedM + 2 || n > 34) fail(kValueError, "random fused passes take 14 to 34 qubits");
    if (count == 0 || count > 4096) fail(kValueError, "count must be between 1 and 4096");
    std::vector<BuiltFusedPass> passes(static_cast<size_t>(count));
    // Each pass draws from its own stream (seed, index), so passes build on pooled workers.
    parallel_for(passes.size(), [&](size_t c) {
        std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + uint64_t(c));
        // Tile qubits: 0 and 1, then ten more drawn by one of four shapes.
        std::vector<int> pool;
        for (int q = kFusedPinned; q < n; q++) pool.push_back(q);
        std::vector<int> T{0, 1};
        const int shape = int(rng() % 4);
        if (shape == 0) {  // uniform
            std::shuffle(pool.begin(), pool.end(), rng);
            T.insert(T.end(), pool.begin(), pool.begin() + (kFusedM - kFusedPinned));
        } else if (shape == 3) {  // one contiguous window
            const int w = kFusedM - kFusedPinned;
            const int start = kFusedPinned + int(rng() % uint64_t(n - kFusedPinned - w + 1));
            for (int q = start; q < start + w; q++) T.push_back(q);
        } else {  // weighted towards low (1) or high (2) qubits
            std::vector<double> wts;
            for (int q : pool) wts.push_back(shape == 1 ? std::pow(0.8, q) : std::pow(0.8, n - 1 - q));
            while (int(T.size()) < kFusedM) {
                std::discrete_distribution<size_t> d(wts.begin(), wts.end());
                const size_t i = d(rng);
                T.push_back(pool[i]);
                wts[i] = 0.0;
            }
        }
        std::sort(T.begin(), T.end());
        // Gates: 1..10 clusters of 4..12 one- and two-qubit gates on five tile qubits each.
        const int clusters = 1 + int(rng() % 10);
        std::vector<Operation> ops;
        for (int b = 0; b < clusters; b++) {
            std::vector<int> five(T);
            std::shuffle(five.begin(), five.end(), rng);
            five.resize(5);
            const int gates = 4 + int(rng() % 9);
            for (int g = 0; g < gates; g++) {
                Operation op;
                if (rng() % 2) {
                    op.type = Operation::One;
                    op.target = uint64_t(five[rng() % 5]);
                    op.m = random_u3(rng);
                } else {
                    const int a = five[rng() % 5];
                    int tq = five[rng() % 5];
                    while (tq == a) tq = five[rng() % 5];
                    op.type = Operation::X;
                    op.target = uint64_t(tq);
                    op.controls.push_back({uint64_t(a), true});
                }
                ops.push_back(op);
            }
        }
        BuiltFusedPass& bp = passes[c];
        bp.src.qubits = T;
        bp.fp = build_fused_pass(ops, T, bp.blocks, bp.upool);
    });
    std::vector<double> ms(passes.size(), -1.0);
    if (measure) {
        PassTimer timer(sim, n);
        for (size_t i = 0; i < passes.size(); i++) ms[i] = timer.time(passes[i]);
    }
    std::string s = "{\"n\": " + std::to_string(n) + ", \"passes\": [";
    for (size_t i = 0; i < passes.size(); i++) s += (i ? ", " : "") + pass_json(n, passes[i].fp, ms[i], -1.0);
    return s + "]}";
}

}  // namespace dq

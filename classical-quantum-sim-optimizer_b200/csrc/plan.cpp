#include "plan.hpp"

#include "cost.hpp"

#include <algorithm>
#include <cstdio>
#include <string>

namespace dq {

Plan::Plan(Simulator& sim, const char* json, size_t len, uint64_t shots) : opt_(sim.options()), shots_(shots) {
    ops_ = compile_json(json, len, &n_, &ncb_);
    if (n_ >= 40) fail(kMemoryError, "State byte size exceeds the device");
    seed_ = opt_.has_seed ? opt_.seed : 0x5eedULL;
    prefix_end_ = ops_.size();
    for (size_t i = 0; i < ops_.size(); i++)
        if (!ops_[i].is_unitary()) {
            prefix_end_ = i;
            break;
        }
    terminal_ = true;
    for (size_t i = prefix_end_; i < ops_.size(); i++)
        if (ops_[i].type != Operation::Measure) terminal_ = false;
    dev_ = sim.ensure_device();
    {
        std::lock_guard<std::mutex> lk(dev_->mu);
        dev_->activate();
        st_.allocate(int(n_), 1, ncb_, opt_.precision == Precision::C64);
    }
    if (terminal_ && prefix_end_ < ops_.size() && shots_ > 0) {
        for (size_t i = prefix_end_; i < ops_.size(); i++) sample_qubits_.push_back(ops_[i].qubit);
        std::sort(sample_qubits_.begin(), sample_qubits_.end());
        sample_qubits_.erase(std::unique(sample_qubits_.begin(), sample_qubits_.end()), sample_qubits_.end());
        std::reverse(sample_qubits_.begin(), sample_qubits_.end());
        const uint64_t clen = uint64_t(1) << sample_qubits_.size();
        cdf_.alloc(clen * 8, "the sampling table");
        tmp_.alloc(k::scan_tmp_size(clen) * 8, "scan scratch");
        idx_.alloc(shots_ * 8, "sampled outcomes");
        scalar_.alloc(16, "sampling total");
    }
    const size_t end = (terminal_ && cdf_.p) ? prefix_end_ : ops_.size();
    ex_ = std::make_unique<Executor>(ops_, 0, end, exec_config(opt_, n_));
    // Upload the matrix pool and warm the kernels once outside any timing.
    run(false);
    const CostModel* model = sim.cost_model();
    ExecConfig lc = exec_config(opt_, n_, false, model);
    if (model && lc.tiled) {
        // Learned plan vs the greedy fixed-width plan: the faster one is kept,
        // and a learned plan slower than greedy is rejected and logged.
        auto learned = std::make_unique<Executor>(ops_, 0, end, lc);
        // A fused-pass model that picks, in every segment, the plan of the hand rule's
        // own cap has chosen the very same plan (the planner is deterministic): nothing
        // to compare, so it is neither timed again nor counted as a rejection.
        bool same = lc.pass_model != nullptr && learned->fused_choices().size() == ex_->fused_choices().size() &&
                    learned->chosen_widths() == ex_->chosen_widths();
        for (size_t s = 0; same && s < learned->fused_choices().size(); s++) {
            const FusedPlanChoice& a = learned->fused_choices()[s];
            const FusedPlanChoice& b = ex_->fused_choices()[s];
            same = a.caps[a.chosen] == b.caps[b.chosen];
        }
        greedy_ms_ = std::min(run(false), run(false));
        std::vector<int> widths = learned->chosen_widths();
        const std::vector<FusedPlanChoice> choices = learned->fused_choices();
        if (same) {
            learned_ms_ = greedy_ms_;
            rejected_ = false;
            used_learned_ = true;
        } else {
            std::swap(ex_, learned);
            run(false);
            learned_ms_ = std::min(run(false), run(false));
            rejected_ = learned_ms_ > greedy_ms_;
            if (rejected_) std::swap(ex_, learned);
            used_learned_ = !rejected_;
        }
        std::string w;
        for (size_t i = 0; i < widths.size(); i++) w += (i ? "," : "") + std::to_string(widths[i]);
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "{\"qubits\": %llu, \"ops\": %llu, \"greedy_ms\": %.4f, \"learned_ms\": %.4f, \"rejected\": %s, ",
                      (unsigned long long)n_, (unsigned long long)ops_.size(), greedy_ms_, learned_ms_,
                      rejected_ ? "true" : "false");
        std::string line = std::string(buf) + "\"same_plan\": " + (same ? "true" : "false") + ", \"kind\": \"" +
                           (model->kind() == kCostFusedPasses ? "fused_passes" : "tile_ops") + "\", \"widths\": [" + w +
                           "], \"fused_plans\": [";
        // Per planned segment: the candidate plans (spread cap, passes, blocks, hand-rule
        // cost, predicted ms), the rule's choice and the model's.
        for (size_t s = 0; s < choices.size(); s++) {
            const FusedPlanChoice& c = choices[s];
            line += s ? ", {" : "{";
            line += "\"rule_choice\": " + std::to_string(c.rule_choice) + ", \"chosen\": " + std::to_string(c.chosen) +
                    ", \"candidates\": [";
            for (size_t i = 0; i < c.caps.size(); i++) {
                std::snprintf(buf, sizeof buf,
                              "%s{\"cap\": %d, \"passes\": %zu, \"blocks\": %zu, \"rule_cost\": %.2f, \"predicted_ms\": %.4f}",
                              i ? ", " : "", c.caps[i], c.passes[i], c.blocks[i], c.rule_cost[i],
                              i < c.predicted_ms.size() ? c.predicted_ms[i] : -1.0);
                line += buf;
            }
            line += "]}";
        }
        sim.log_planner(line + "]}");
    }
}

double Plan::state_bytes() const { return double(uint64_t(1) << n_) * (st_.c64 ? 8.0 : 16.0); }

double Plan::run(bool record) {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cudaStream_t s = dev_->stream;
    EventRecorder rec(s);
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "cudaEventCreate");
    cuda_check(cudaEventCreate(&b), "cudaEventCreate");
    cuda_check(cudaEventRecord(a, s), "cudaEventRecord");
    k::Batch bt = st_.view(s, 1);
    // |0...0>: written here, or built by a first fused pass in its tiles.
    const bool built = ex_->starts_with_fused_pass();
    if (!built) k::init_basis(bt);
    cuda_check(cudaMemsetAsync(st_.cbits.p, 0, size_t(st_.cwords) * 8, s), "clear cbits");
    cuda_check(cudaMemsetAsync(st_.draws.p, 0, 8, s), "clear draws");
    cuda_check(cudaMemsetAsync(st_.err.p, 0, 16, s), "clear error flag");
    cuda_check(cudaMemcpyAsync(st_.seeds.p, &seed_, 8, cudaMemcpyHostToDevice, s), "seed");
    ex_->run(bt, nullptr, record ? &rec : nullptr, /*normalize=*/cdf_.p == nullptr, /*from_basis=*/built);
    if (cdf_.p) {
        const uint64_t clen = uint64_t(1) << sample_qubits_.size();
        bool full = sample_qubits_.size() == n_;
        for (uint64_t t = 0; full && t < n_; t++) full = sample_qubits_[t] == n_ - 1 - t;
        // State read once and two-level running sums written once (the sampler adds
        // each probed entry's tile offset itself).
        const int scans = k::scan_launches(clen) - (clen > 2048 ? 1 : 0);
        if (record)
            rec.begin(kcSample, double(uint64_t(1) << n_) * (st_.c64 ? 8.0 : 16.0) + 8.0 * clen,
                      scans + (full ? 0 : 1) + 2);
        if (full) {
            k::scan_probs(bt, cdf_.as<double>(), tmp_.as<double>(), false);
        } else {
            std::vector<int> q(sample_qubits_.begin(), sample_qubits_.end());
            k::marginal(bt, q, cdf_.as<double>());
            k::scan_local(s, cdf_.as<double>(), clen, tmp_.as<double>());
        }
        k::take_total(s, cdf_.as<double>(), clen, tmp_.as<double>(), scalar_.as<double>(), st_.err.as<int>());
        k::sample_sums(s, cdf_.as<double>(), tmp_.as<double>(), clen, scalar_.as<double>(), 0.0, false, seed_,
                       shots_, true, idx_.as<uint64_t>());
        if (record) rec.end();
    }
    cuda_check(cudaEventRecord(b, s), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(b), "cudaEventSynchronize");
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, a, b), "cudaEventElapsedTime");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (record) rec.collect(ms_, launches_, bytes_);
    int flag = 0;
    cuda_check(cudaMemcpy(&flag, st_.err.p, sizeof(int), cudaMemcpyDeviceToHost), "read error flag");
    if (flag == 3) fail(kRuntimeError, "a tensor-core pass gave up on a bounded wait");
    if (flag) fail(kRuntimeError, "Cannot measure or sample a state with nonfinite or zero norm");
    return double(ms);
}

void Plan::stats(double* ms, uint64_t* launches, double* bytes) const {
    for (int c = 0; c < kcNumClasses; c++) {
        ms[c] = ms_[c];
        launches[c] = launches_[c];
        bytes[c] = bytes_[c];
    }
}

void Plan::statevector(double* out) const {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    const uint64_t len = uint64_t(1) << n_;
    if (!st_.c64) {
        cuda_check(cudaMemcpy(out, st_.amps.p, len * 16, cudaMemcpyDeviceToHost), "read state");
        return;
    }
    std::vector<float> tmp(len * 2);
    cuda_check(cudaMemcpy(tmp.data(), st_.amps.p, len * 8, cudaMemcpyDeviceToHost), "read state");
    for (uint64_t i = 0; i < 2 * len; i++) out[i] = double(tmp[i]);
}

void Plan::compare(const Plan& other, double* fidelity, double* max_abs_err) const {
    if (other.n_ != n_) fail(kValueError, "plans have different qubit counts");
    if (other.dev_->ordinal != dev_->ordinal) fail(kValueError, "plans live on different devices");
    std::lock_guard<std::mutex> lk(dev_->mu);
    std::unique_lock<std::mutex> lk2(other.dev_->mu, std::defer_lock);
    if (other.dev_ != dev_) lk2.lock();
    dev_->activate();
    cuda_check(cudaStreamSynchronize(other.dev_->stream), "stream synchronize");
    DevMem part;
    part.alloc(size_t(k::kDotBlocks) * 5 * 8, "comparison partial sums");
    k::compare(dev_->stream, st_.amps.p, st_.c64, other.st_.amps.p, other.st_.c64, uint64_t(1) << n_,
               part.as<double>());
    std::vector<double> h(size_t(k::kDotBlocks) * 5);
    cuda_check(cudaMemcpyAsync(h.data(), part.p, h.size() * 8, cudaMemcpyDeviceToHost, dev_->stream), "read");
    dev_->sync();
    double re = 0, im = 0, mx = 0, na = 0, nb = 0;
    for (int i = 0; i < k::kDotBlocks; i++) {
        re += h[i * 5];
        im += h[i * 5 + 1];
        mx = std::max(mx, h[i * 5 + 2]);
        na += h[i * 5 + 3];
        nb += h[i * 5 + 4];
    }
    // |<a|b>|^2 / (<a|a> <b|b>): a sampling run leaves the fused form's last
    // pass unrescaled (sampling divides by the total), so norms are divided out.
    *fidelity = (re * re + im * im) / (na * nb);
    *max_abs_err = mx;
}

void Plan::record_costs(std::vector<float>& X, std::vector<float>& y) {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    k::Batch bt = st_.view(dev_->stream, 1);
    ex_->record_costs(bt, X, y);
}

void Plan::samples(uint64_t* out) const {
    if (!idx_.p) fail(kValueError, "the circuit has no terminal measurements to sample");
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cuda_check(cudaMemcpy(out, idx_.p, shots_ * 8, cudaMemcpyDeviceToHost), "read samples");
}

}  // namespace dq

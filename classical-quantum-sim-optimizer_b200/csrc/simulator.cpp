#include "simulator.hpp"

#include "cost.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>

namespace dq {
namespace {

using clk = std::chrono::steady_clock;
double since(clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); }

// Sorts sampled outcomes ascending: LSD radix sort on 16-bit digits, only as
// many passes as the largest value needs (std::sort below 4096 values).
void sort_outcomes(std::vector<uint64_t>& v) {
    if (v.size() < 4096) {
        std::sort(v.begin(), v.end());
        return;
    }
    uint64_t top = 0;
    for (uint64_t x : v) top |= x;
    std::vector<uint64_t> tmp(v.size());
    std::vector<size_t> start(65537);
    for (int shift = 0; shift < 64 && (top >> shift) != 0; shift += 16) {
        std::fill(start.begin(), start.end(), size_t(0));
        for (uint64_t x : v) start[((x >> shift) & 0xffff) + 1]++;
        for (size_t d = 0; d < 65536; d++) start[d + 1] += start[d];
        for (uint64_t x : v) tmp[start[(x >> shift) & 0xffff]++] = x;
        v.swap(tmp);
    }
}

// state_layout, shots.rs:22-31, for `amp` bytes per amplitude.
void state_layout(uint64_t n, uint64_t amp, uint64_t* len, uint64_t* bytes) {
    if (n >= 64) fail(kMemoryError, "State dimension overflow");
    *len = uint64_t(1) << n;
    unsigned __int128 b = (unsigned __int128)(*len) * amp;
    if (b > kIsizeMax) fail(kMemoryError, "State byte size overflow");
    *bytes = uint64_t(b);
}

// check_budget, shots.rs:43-48
void check_budget(uint64_t required, uint64_t budget) {
    if (required > budget)
        fail(kMemoryError, "Simulation needs at least " + std::to_string(required) +
                               " working bytes, exceeding max_memory_mb budget (" + std::to_string(budget) + " bytes)");
}

// format_bits, shots.rs:50-56: cbit 0 is the rightmost character.
std::string format_bits(const uint8_t* cbits, uint64_t ncb) {
    std::string s(ncb, '0');
    for (uint64_t i = 0; i < ncb; i++) s[ncb - 1 - i] = char('0' + cbits[i]);
    return s;
}

void upload_u64(void* dst, const std::vector<uint64_t>& v, cudaStream_t s) {
    cuda_check(cudaMemcpyAsync(dst, v.data(), v.size() * 8, cudaMemcpyHostToDevice, s), "upload");
}

void check_err_flag(const StateBatch& st, cudaStream_t s) {
    int flag = 0;
    cuda_check(cudaMemcpyAsync(&flag, st.err.p, sizeof(int), cudaMemcpyDeviceToHost, s), "read error flag");
    cuda_check(cudaStreamSynchronize(s), "stream synchronize");
    if (flag == 3) fail(kRuntimeError, "a tensor-core pass gave up on a bounded wait");
    if (flag) fail(kRuntimeError, "Cannot measure a state with nonfinite or zero norm");
}

void reset_bookkeeping(const StateBatch& st, uint64_t W, const std::vector<uint64_t>& seeds, cudaStream_t s) {
    cuda_check(cudaMemsetAsync(st.cbits.p, 0, size_t(W) * st.cwords * 8, s), "clear cbits");
    cuda_check(cudaMemsetAsync(st.draws.p, 0, size_t(W) * 8, s), "clear draws");
    cuda_check(cudaMemsetAsync(st.err.p, 0, 16, s), "clear error flag");
    upload_u64(st.seeds.p, seeds, s);
}

bool is_full_descending(const std::vector<uint64_t>& q, uint64_t n) {
    if (q.size() != n) return false;
    for (uint64_t t = 0; t < n; t++)
        if (q[t] != n - 1 - t) return false;
    return true;
}

// Probabilities of state 0 over `qubits` into a device buffer of 2^k doubles.
void probs_to(const k::Batch& b, const std::vector<uint64_t>& qubits, double* out) {
    if (is_full_descending(qubits, uint64_t(b.n))) {
        k::norm2(b, out);
    } else {
        std::vector<int> q;
        for (auto x : qubits) q.push_back(int(x));
        k::marginal(b, q, out);
    }
}

// Two-level running sums of state 0's probabilities over `qubits` on the
// device (sums within 2048-entry tiles in cdf, inclusive sums of whole tiles in
// tmp; the full register in descending order reads the state directly);
// returns the total, the last entry of the full running sums.
double build_sums(const k::Batch& b, const std::vector<uint64_t>& qubits, double* cdf, uint64_t len, DevMem& tmp) {
    cudaStream_t s = b.stream;
    tmp.ensure_on(k::scan_tmp_size(len) * 8, s, "scan scratch");
    if (is_full_descending(qubits, uint64_t(b.n))) {
        k::scan_probs(b, cdf, tmp.as<double>(), false);
    } else {
        probs_to(b, qubits, cdf);
        k::scan_local(s, cdf, len, tmp.as<double>());
    }
    double last = 0, offset = 0;
    const uint64_t t = k::scan_tile_of(len - 1);
    cuda_check(cudaMemcpyAsync(&last, cdf + (len - 1), 8, cudaMemcpyDeviceToHost, s), "read total");
    if (t > 0) cuda_check(cudaMemcpyAsync(&offset, tmp.as<double>() + (t - 1), 8, cudaMemcpyDeviceToHost, s), "read total");
    cuda_check(cudaStreamSynchronize(s), "stream synchronize");
    return t > 0 ? last + offset : last;
}

std::string json_double(double v) {
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    std::string s(buf);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return s;
}

}  // namespace

ExecConfig exec_config(const Options& o, uint64_t n, bool force_per_gate, const CostModel* model) {
    ExecConfig c;
    if (model && model->kind() == kCostFusedPasses)
        c.pass_model = model;
    else
        c.model = model;
    c.c64 = o.precision == Precision::C64;
    c.tiled = !force_per_gate && o.execution != 1;
    c.tile_m = o.tile_qubits > 0 ? o.tile_qubits : (c.c64 ? 13 : 12);
    c.fuse = o.fusion_width > 0 ? o.fusion_width : 2;
    // complex64 runs its tile passes as fused 5-qubit tensor-core blocks unless a
    // CUDA-core tile shape or a narrower fusion width is asked for.
    c.fused = c.c64 && c.tiled && (o.fusion_width == 5 || (o.fusion_width == 0 && o.tile_qubits == 0));
    c.n = int(n);
    return c;
}

std::vector<Operation> compile_json(const char* json, size_t len, uint64_t* n, uint64_t* ncb) {
    Circuit c = parse_circuit(json, len);
    validate_circuit(c);
    if (n) *n = c.num_qubits();
    if (ncb) *ncb = c.num_cbits();
    return compile(c.instructions);
}

Simulator::Simulator(const Options& o) : opt_(o) {
    // simulator.rs:234-246
    if (o.max_memory_mb == 0 || o.max_memory_mb > kIsizeMax / (1024 * 1024))
        fail(kValueError, "max_memory_mb must be positive and representable in bytes");
    if (o.has_max_parallel_shots && o.max_parallel_shots == 0)
        fail(kValueError, "max_parallel_shots must be positive or None");
    budget_ = o.max_memory_mb * 1024 * 1024;
}

Simulator::~Simulator() {
    if (ws_ && dev_) {
        std::lock_guard<std::mutex> lk(dev_->mu);
        cudaSetDevice(dev_->ordinal);
        ws_.reset();
    }
}

uint64_t Simulator::next_seed() {
    if (opt_.has_seed) return opt_.seed;
    std::random_device rd;
    return (uint64_t(rd()) << 32) ^ uint64_t(rd());
}

ShotOutput Simulator::simulate_shots(const char* json, size_t len, uint64_t shots, bool profile, double* pre,
                                     double* fus) {
    auto total0 = clk::now();
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (double& v : phases_) v = 0.0;
    }
    profile = profile || opt_.profile;
    std::shared_ptr<ShotPlan> plan;
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (size_t i = 0; i < plans_.size(); i++)
            if (plans_[i]->json.size() == len && std::memcmp(plans_[i]->json.data(), json, len) == 0) {
                plan = plans_[i];
                plans_.erase(plans_.begin() + long(i));
                plans_.insert(plans_.begin(), plan);
                break;
            }
    }
    double preprocessing = 0.0, fusion = 0.0;
    if (!plan) {
        Circuit c = parse_circuit(json, len);
        validate_circuit(c);
        preprocessing = since(total0);
        auto f0 = clk::now();
        plan = std::make_shared<ShotPlan>();
        plan->ops = compile(c.instructions);
        fusion = since(f0);
        plan->json.assign(json, len);
        plan->n = c.num_qubits();
        plan->ncb = c.num_cbits();
        std::lock_guard<std::mutex> lk(mu_);
        plans_.insert(plans_.begin(), plan);
        if (plans_.size() > kShotPlans) plans_.resize(kShotPlans);
    }
    set_phase(kPhParse, preprocessing);
    set_phase(kPhCompile, fusion);
    uint64_t seed = next_seed();
    auto s0 = clk::now();
    ShotOutput out = run_shots(plan->ops, plan->n, plan->ncb, shots, seed, profile, plan.get());
    double shots_total = since(s0);
    set_phase(kPhTotal, since(total0));
    if (pre) *pre = preprocessing;
    if (fus) *fus = fusion;
    if (profile) write_shots_profile(out, preprocessing, fusion, shots_total, since(total0), shots);
    return out;
}

ShotOutput Simulator::run_shots(const std::vector<Operation>& ops, uint64_t n, uint64_t ncb, uint64_t shots,
                                uint64_t seed, bool profile, ShotPlan* shot_plan) {
    ShotOutput out;
    if (shots == 0) {
        out.strategy = "empty";
        return out;
    }
    const uint64_t amp = opt_.precision == Precision::C64 ? 8 : 16;
    uint64_t len, state_bytes;
    state_layout(n, amp, &len, &state_bytes);
    if (state_bytes > kU64Max - ncb) fail(kMemoryError, "Working memory size overflow");
    const uint64_t worker_bytes = state_bytes + ncb;
    check_budget(worker_bytes, budget_);
    size_t prefix_end = ops.size();
    for (size_t i = 0; i < ops.size(); i++)
        if (!ops[i].is_unitary()) {
            prefix_end = i;
            break;
        }
    bool terminal = true;
    for (size_t i = prefix_end; i < ops.size(); i++)
        if (ops[i].type != Operation::Measure) terminal = false;
    const bool c64 = opt_.precision == Precision::C64;

    if (opt_.sample_terminal && terminal) {
        std::map<uint64_t, uint64_t> mapping;  // cbit -> qubit; the last write wins
        for (size_t i = prefix_end; i < ops.size(); i++) mapping[ops[i].cbit] = ops[i].qubit;
        if (mapping.empty()) {
            out.strategy = "terminal_sampling";
            out.counts[std::string(ncb, '0')] = shots;
            return out;
        }
        std::vector<uint64_t> qubits;
        for (auto& kv : mapping) qubits.push_back(kv.second);
        std::sort(qubits.begin(), qubits.end());
        qubits.erase(std::unique(qubits.begin(), qubits.end()), qubits.end());
        std::reverse(qubits.begin(), qubits.end());
        const uint64_t kq = qubits.size();
        std::vector<std::pair<uint64_t, uint64_t>> shifts;  // (cbit, shift)
        for (auto& kv : mapping) {
            uint64_t pos = uint64_t(std::find(qubits.begin(), qubits.end(), kv.second) - qubits.begin());
            shifts.emplace_back(kv.first, kq - 1 - pos);
        }
        if (kq >= 61) fail(kMemoryError, "Sampling memory overflow");
        const uint64_t cdf_bytes = (uint64_t(1) << kq) * 8;
        if (worker_bytes <= kU64Max - cdf_bytes && worker_bytes + cdf_bytes <= budget_) {
            const uint64_t required = worker_bytes + cdf_bytes;
            ensure_device();
            std::lock_guard<std::mutex> lk(dev_->mu);
            dev_->activate();
            cudaStream_t s = dev_->stream;
            uint64_t kept_seed = seed;
            clk::time_point mark = clk::now();
            auto phase = [&](int i) {
                const clk::time_point now = clk::now();
                set_phase(i, std::chrono::duration<double>(now - mark).count());
                mark = now;
            };
            {
                // The workspace of the previous call is reused where its sizes match.
                if (!ws_) ws_ = std::make_unique<SamplingWorkspace>();
                StateBatch& st = ws_->st;
                if (!st.amps.p || st.n != int(n) || st.W != 1 || st.ncb != ncb || st.c64 != c64)
                    st.allocate(int(n), 1, ncb, c64, s);
                k::Batch b = st.view(s, 1);
                reset_bookkeeping(st, 1, {kept_seed}, s);
                phase(kPhState);
                DevMem& cdf = ws_->table;
                DevMem& tmp = ws_->scratch;
                DevMem& idx = ws_->outcomes;
                const uint64_t clen = uint64_t(1) << kq;
                if (cdf.bytes != clen * 8) cdf.alloc_on(clen * 8, s, "the sampling table");
                const uint64_t tmp_bytes = std::max<uint64_t>(k::scan_tmp_size(clen) * 8, 16);
                if (tmp.bytes != tmp_bytes) tmp.alloc_on(tmp_bytes, s, "scan scratch");
                if (idx.bytes != shots * 8) idx.alloc_on(shots * 8, s, "sampled outcomes");
                phase(kPhTable);
                // The prefix's executor: kept with the circuit's cached plan (the
                // device lock above serialises its use), or built for this call.
                std::unique_ptr<Executor> own;
                Executor* ex = shot_plan ? shot_plan->prefix.get() : nullptr;
                if (!ex) {
                    own = std::make_unique<Executor>(ops, 0, prefix_end, exec_config(opt_, n));
                    ex = own.get();
                    if (shot_plan) shot_plan->prefix = std::move(own);
                }
                phase(kPhPlan);
                // Device time of the prefix, read once the sums below have synchronised.
                cudaEvent_t ev[2] = {nullptr, nullptr};
                for (cudaEvent_t& e : ev) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
                struct EventPair {
                    cudaEvent_t* e;
                    ~EventPair() {
                        for (int i = 0; i < 2; i++) cudaEventDestroy(e[i]);
                    }
                } ev_guard{ev};
                cuda_check(cudaEventRecord(ev[0], s), "cudaEventRecord");
                // |0...0>: written here, or built by a first fused pass in its tiles.
                const bool built = ex->starts_with_fused_pass();
                if (!built) k::init_basis(b);
                ex->run(b, nullptr, nullptr, /*normalize=*/false, /*from_basis=*/built);  // the sampler divides by the total
                cuda_check(cudaEventRecord(ev[1], s), "cudaEventRecord");
                phase(kPhRun);
                double total = build_sums(b, qubits, cdf.as<double>(), clen, tmp);
                if (!std::isfinite(total) || total <= 0.0) fail(kMemoryError, "Invalid state normalization when sampling");
                phase(kPhSums);
                float prefix_ms = 0.f;
                if (cudaEventElapsedTime(&prefix_ms, ev[0], ev[1]) == cudaSuccess)
                    set_phase(kPhPrefixDevice, double(prefix_ms) * 1e-3);
                k::sample_sums(s, cdf.as<double>(), tmp.as<double>(), clen, nullptr, total, false, seed, shots, true,
                               idx.as<uint64_t>());
                std::vector<uint64_t> h(shots);
                cuda_check(cudaMemcpyAsync(h.data(), idx.p, shots * 8, cudaMemcpyDeviceToHost, s), "read samples");
                cuda_check(cudaStreamSynchronize(s), "stream synchronize");
                phase(kPhSample);
                sort_outcomes(h);
                if (ncb <= 64) {
                    // Classical-register value of each distinct outcome, merged by value.
                    // Where every cbit reads the sampled bit of its own position the
                    // value is the outcome masked to those bits.
                    bool same_bit = true;
                    uint64_t same_mask = 0;
                    for (auto& sh : shifts) {
                        same_bit = same_bit && sh.first == sh.second;
                        same_mask |= uint64_t(1) << sh.second;
                    }
                    std::vector<std::pair<uint64_t, uint64_t>> kc;
                    for (size_t i = 0; i < h.size();) {
                        size_t j = i;
                        while (j < h.size() && h[j] == h[i]) j++;
                        uint64_t key = 0;
                        if (same_bit)
                            key = h[i] & same_mask;
                        else
                            for (auto& sh : shifts) key |= ((h[i] >> sh.second) & 1) << sh.first;
                        kc.emplace_back(key, uint64_t(j - i));
                        i = j;
                    }
                    if (!std::is_sorted(kc.begin(), kc.end())) std::sort(kc.begin(), kc.end());
                    size_t distinct = 0;
                    for (size_t i = 0; i < kc.size(); i++) {
                        if (distinct && kc[i].first == kc[distinct - 1].first)
                            kc[distinct - 1].second += kc[i].second;
                        else
                            kc[distinct++] = kc[i];
                    }
                    out.key_width = ncb;
                    out.flat_keys.assign(distinct * ncb, '0');
                    out.flat_counts.resize(distinct);
                    // cbit 0 is the rightmost character; whole bytes of the value through
                    // a table of their eight characters (most significant bit first).
                    static const std::array<std::array<char, 8>, 256> byte_chars = [] {
                        std::array<std::array<char, 8>, 256> t{};
                        for (int v = 0; v < 256; v++)
                            for (int b = 0; b < 8; b++) t[size_t(v)][size_t(7 - b)] = char('0' + ((v >> b) & 1));
                        return t;
                    }();
                    char* key = &out.flat_keys[0];
                    for (size_t i = 0; i < distinct; i++, key += ncb) {
                        const uint64_t v = kc[i].first;
                        uint64_t c = 0;
                        for (; c + 8 <= ncb; c += 8)  // cbits c..c+7 end at character ncb - 1 - c
                            std::memcpy(key + (ncb - 8 - c), byte_chars[size_t((v >> c) & 0xFFu)].data(), 8);
                        for (; c < ncb; c++) key[ncb - 1 - c] = char('0' + ((v >> c) & 1));
                        out.flat_counts[i] = kc[i].second;
                    }
                } else {
                    std::vector<uint8_t> cb(ncb, 0);
                    for (size_t i = 0; i < h.size();) {
                        size_t j = i;
                        while (j < h.size() && h[j] == h[i]) j++;
                        for (auto& sh : shifts) cb[sh.first] = uint8_t((h[i] >> sh.second) & 1);
                        out.counts[format_bits(cb.data(), ncb)] += uint64_t(j - i);
                        i = j;
                    }
                }
                phase(kPhKeys);
            }
            phase(kPhRelease);
            out.strategy = "terminal_sampling";
            out.parallel_shots = 1;
            out.working_bytes = required;
            out.prefix_ops = prefix_end;
            return out;
        }
        // Fall back to trajectories when the sampling table exceeds the budget.
    }

    const bool cache_prefix = shots > 1 && prefix_end > 0 && state_bytes <= budget_ - worker_bytes;
    const uint64_t prefix_bytes = cache_prefix ? state_bytes : 0;
    // The device's concurrent-trajectory cap plays the role of Rayon's thread
    // count: at most 65536 states, and no more than 2^28 amplitudes per batch.
    const uint64_t cap = std::max<uint64_t>(1, std::min<uint64_t>(65536, (uint64_t(1) << 28) >> std::min<uint64_t>(n, 28)));
    uint64_t workers = std::min(shots, opt_.has_max_parallel_shots ? opt_.max_parallel_shots : cap);
    workers = std::min(workers, cap);
    workers = std::min(workers, (budget_ - prefix_bytes) / worker_bytes);
    workers = std::max<uint64_t>(workers, 1);

    ensure_device();
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cudaStream_t s = dev_->stream;
    StateBatch prefix;
    if (cache_prefix) {
        prefix.allocate(int(n), 1, ncb, c64);
        k::Batch pb = prefix.view(s, 1);
        k::init_basis(pb);
        reset_bookkeeping(prefix, 1, {seed}, s);
        Executor pre(ops, 0, prefix_end, exec_config(opt_, n));
        pre.run(pb, nullptr);
    }
    StateBatch st;
    st.allocate(int(n), workers, ncb, c64);
    Executor ex(ops, cache_prefix ? prefix_end : 0, ops.size(), exec_config(opt_, n));
    if (profile) out.shot_times.assign(shots, 0.0);
    std::vector<uint64_t> hbits(size_t(workers) * st.cwords);
    std::vector<uint8_t> cb(ncb);
    for (uint64_t r0 = 0; r0 < shots; r0 += workers) {
        const uint64_t Wr = std::min(workers, shots - r0);
        auto t0 = clk::now();
        k::Batch b = st.view(s, Wr);
        if (cache_prefix)
            k::broadcast(b, prefix.amps.p);
        else
            k::init_basis(b);
        std::vector<uint64_t> seeds(Wr);
        for (uint64_t i = 0; i < Wr; i++) seeds[i] = seed + r0 + i;  // wrapping, shots.rs:224
        reset_bookkeeping(st, Wr, seeds, s);
        ex.run(b, nullptr);
        cuda_check(cudaMemcpyAsync(hbits.data(), st.cbits.p, size_t(Wr) * st.cwords * 8, cudaMemcpyDeviceToHost, s),
                   "read classical bits");
        check_err_flag(st, s);
        for (uint64_t i = 0; i < Wr; i++) {
            const uint64_t* w = hbits.data() + i * st.cwords;
            for (uint64_t c = 0; c < ncb; c++) cb[c] = uint8_t((w[c >> 6] >> (c & 63)) & 1);
            out.counts[format_bits(cb.data(), ncb)]++;
        }
        if (profile) {
            double per = since(t0) / double(Wr);
            for (uint64_t i = 0; i < Wr; i++) out.shot_times[r0 + i] = per;
        }
    }
    out.strategy = "trajectories";
    out.parallel_shots = workers;
    out.working_bytes = prefix_bytes + workers * worker_bytes;
    out.prefix_ops = cache_prefix ? prefix_end : 0;
    return out;
}

std::unique_ptr<Result> Simulator::simulate(const char* json, size_t len) {
    auto total0 = clk::now();
    Circuit c = parse_circuit(json, len);
    validate_circuit(c);
    const uint64_t n = c.num_qubits(), ncb = c.num_cbits();
    const uint64_t amp = opt_.precision == Precision::C64 ? 8 : 16;
    uint64_t slen, bytes;
    state_layout(n, amp, &slen, &bytes);
    if (bytes > kU64Max - ncb) fail(kMemoryError, "Working memory size overflow");
    check_budget(bytes + ncb, budget_);
    std::vector<Operation> plan = compile(c.instructions);
    uint64_t seed = next_seed();
    ensure_device();
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cudaStream_t s = dev_->stream;
    auto res = std::make_unique<Result>();
    res->dev = dev_;
    res->n = n;
    res->state.allocate(int(n), 1, ncb, opt_.precision == Precision::C64);
    k::Batch b = res->state.view(s, 1);
    k::init_basis(b);
    reset_bookkeeping(res->state, 1, {seed}, s);
    // Profiling times each reference operation, so it runs the per-gate form.
    Executor ex(plan, 0, plan.size(), exec_config(opt_, n, opt_.profile));
    ProfileAcc acc;
    ex.run(b, opt_.profile ? &acc : nullptr);
    check_err_flag(res->state, s);
    std::vector<uint64_t> hbits(res->state.cwords);
    cuda_check(cudaMemcpyAsync(hbits.data(), res->state.cbits.p, hbits.size() * 8, cudaMemcpyDeviceToHost, s),
               "read classical bits");
    cuda_check(cudaStreamSynchronize(s), "stream synchronize");
    res->cbits.resize(ncb);
    for (uint64_t i = 0; i < ncb; i++) res->cbits[i] = uint8_t((hbits[i >> 6] >> (i & 63)) & 1);
    if (opt_.profile) {
        res->profile.present = true;
        res->profile.acc = acc;
        res->profile.total_time = since(total0);
    }
    return res;
}

void Result::statevector(double* out) const {
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    const uint64_t len = uint64_t(1) << n;
    if (!state.c64) {
        cuda_check(cudaMemcpyAsync(out, state.amps.p, len * 16, cudaMemcpyDeviceToHost, dev->stream), "read state");
        dev->sync();
        return;
    }
    std::vector<float> tmp(len * 2);
    cuda_check(cudaMemcpyAsync(tmp.data(), state.amps.p, len * 8, cudaMemcpyDeviceToHost, dev->stream), "read state");
    dev->sync();
    for (uint64_t i = 0; i < 2 * len; i++) out[i] = double(tmp[i]);
}

void Result::probabilities(const std::vector<uint64_t>& qubits, double* out) const {
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    const uint64_t m = uint64_t(1) << qubits.size();
    DevMem buf;
    buf.alloc(m * 8, "probabilities");
    k::Batch b = state.view(dev->stream, 1);
    probs_to(b, qubits, buf.as<double>());
    cuda_check(cudaMemcpyAsync(out, buf.p, m * 8, cudaMemcpyDeviceToHost, dev->stream), "read probabilities");
    dev->sync();
}

std::unordered_map<uint64_t, uint64_t> Result::counts(uint64_t shots, const std::vector<uint64_t>& qubits,
                                                      uint64_t seed) const {
    std::unordered_map<uint64_t, uint64_t> res;
    if (shots == 0) return res;
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    cudaStream_t s = dev->stream;
    const uint64_t m = uint64_t(1) << qubits.size();
    DevMem cdf, tmp, idx;
    cdf.alloc(m * 8, "the sampling table");
    k::Batch b = state.view(s, 1);
    double total = build_sums(b, qubits, cdf.as<double>(), m, tmp);
    if (!std::isfinite(total) || total <= 0.0) fail(kRuntimeError, "Cannot sample a state with nonfinite or zero norm");
    idx.alloc(shots * 8, "sampled outcomes");
    k::sample_sums(s, cdf.as<double>(), tmp.as<double>(), m, nullptr, total, true, seed, shots, false,
                   idx.as<uint64_t>());
    std::vector<uint64_t> h(shots);
    cuda_check(cudaMemcpyAsync(h.data(), idx.p, shots * 8, cudaMemcpyDeviceToHost, s), "read samples");
    dev->sync();
    for (uint64_t v : h) res[v]++;
    return res;
}

double Result::fidelity(const double* other, uint64_t len) const {
    if (len != (uint64_t(1) << n)) return 0.0;
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    DevMem o, part;
    o.alloc(len * 16, "fidelity operand");
    part.alloc(k::kDotBlocks * 16, "fidelity partial sums");
    cuda_check(cudaMemcpyAsync(o.p, other, len * 16, cudaMemcpyHostToDevice, dev->stream), "upload operand");
    k::Batch b = state.view(dev->stream, 1);
    int nb = k::dot_partials(b, o.as<double2>(), part.as<double2>());
    std::vector<double2> hp(nb);
    cuda_check(cudaMemcpyAsync(hp.data(), part.p, nb * 16, cudaMemcpyDeviceToHost, dev->stream), "read partials");
    dev->sync();
    double re = 0, im = 0;
    for (auto& v : hp) {
        re += v.x;
        im += v.y;
    }
    return re * re + im * im;
}

void Result::amplitudes(const uint64_t* indices, uint64_t count, double* out) const {
    const uint64_t len = uint64_t(1) << n;
    for (uint64_t j = 0; j < count; j++)
        if (indices[j] >= len) fail(kValueError, "amplitude index out of range");
    if (count == 0) return;
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    DevMem idx, buf;
    idx.alloc(count * 8, "amplitude indices");
    buf.alloc(count * 16, "amplitudes");
    cuda_check(cudaMemcpyAsync(idx.p, indices, count * 8, cudaMemcpyHostToDevice, dev->stream), "upload indices");
    k::Batch b = state.view(dev->stream, 1);
    k::gather(b, idx.as<uint64_t>(), count, buf.as<double2>());
    cuda_check(cudaMemcpyAsync(out, buf.p, count * 16, cudaMemcpyDeviceToHost, dev->stream), "read amplitudes");
    dev->sync();
}

void Result::pauli_xz(uint64_t x, uint64_t z, double* re, double* im) const {
    const uint64_t len = uint64_t(1) << n;
    if (x >= len || z >= len) fail(kValueError, "Pauli masks exceed the register");
    std::lock_guard<std::mutex> lk(dev->mu);
    dev->activate();
    DevMem part;
    part.alloc(k::kDotBlocks * 16, "expectation partial sums");
    k::Batch b = state.view(dev->stream, 1);
    const int nb = k::pauli_partials(b, x, z, part.as<double2>());
    std::vector<double2> hp(static_cast<size_t>(nb));
    cuda_check(cudaMemcpyAsync(hp.data(), part.p, size_t(nb) * 16, cudaMemcpyDeviceToHost, dev->stream),
               "read partials");
    dev->sync();
    double r = 0, i = 0;
    for (auto& v : hp) {  // fixed order: deterministic
        r += v.x;
        i += v.y;
    }
    *re = r;
    *im = i;
}

void write_shots_profile(const ShotOutput& out, double preprocessing, double fusion, double shots_total, double total,
                         uint64_t shots) {
    ::mkdir("dqsim_profiles", 0777);
    struct stat stt;
    if (::stat("dqsim_profiles", &stt) != 0 || !S_ISDIR(stt.st_mode))
        fail(kRuntimeError, "Failed to write shots profile: cannot create dqsim_profiles");
    auto ns = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::system_clock::now().time_since_epoch())
                  .count();
    std::string path = "dqsim_profiles/statevector_shots_profile_" + std::to_string(ns) + ".json";
    std::string j = "{\n";
    j += "  \"preprocessing_time\": " + json_double(preprocessing) + ",\n";
    j += "  \"fusion_time\": " + json_double(fusion) + ",\n";
    j += "  \"shots_total_time\": " + json_double(shots_total) + ",\n";
    j += "  \"total_time\": " + json_double(total) + ",\n";
    j += "  \"num_shots\": " + std::to_string(shots) + ",\n";
    j += "  \"shot_times\": [";
    for (size_t i = 0; i < out.shot_times.size(); i++) j += (i ? ", " : "") + json_double(out.shot_times[i]);
    j += "],\n";
    j += "  \"execution_strategy\": \"" + out.strategy + "\",\n";
    j += "  \"parallel_shots\": " + std::to_string(out.parallel_shots) + ",\n";
    j += "  \"working_bytes\": " + std::to_string(out.working_bytes) + ",\n";
    j += "  \"deterministic_prefix_ops\": " + std::to_string(out.prefix_ops) + "\n}";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) fail(kRuntimeError, "Failed to write shots profile: cannot open " + path);
    size_t w = std::fwrite(j.data(), 1, j.size(), f);
    std::fclose(f);
    if (w != j.size()) fail(kRuntimeError, "Failed to write shots profile: short write");
}

}  // namespace dq

// extern "C" layer: exceptions become status codes plus a thread-local message.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

#include "../../include/dqsim_sv.h"
#include "batch.hpp"
#include "blocks.hpp"
#include "cost.hpp"
#include "plan.hpp"
#include "portfolio.hpp"
#include "simulator.hpp"

using namespace dq;

namespace dq {
double fp64_fma_tflops(int device);
void measure_noalloc(void* states, int precision, uint64_t num_states, uint64_t num_qubits, uint64_t qubit, int reset,
                     const uint64_t* seeds, const uint64_t* draw_index, int* outcomes);
}

struct dq_plan {
    std::unique_ptr<Plan> impl;
};
struct dq_batch {
    std::unique_ptr<BatchRun> impl;
};
struct dq_cost_model {
    std::unique_ptr<CostModel> impl;
};
struct dq_blocks {
    std::unique_ptr<BlockContext> impl;
};

struct dq_sim {
    std::unique_ptr<Simulator> impl;
};
struct dq_result {
    std::unique_ptr<Result> impl;
};
struct dq_counts {
    uint64_t width = 0;
    std::string keys;  // distinct keys of `width` characters back to back
    std::vector<uint64_t> counts;
};

namespace {
thread_local std::string g_error;

template <typename F>
int guard(F&& f) {
    try {
        g_error.clear();
        f();
        return DQ_OK;
    } catch (const Error& e) {
        g_error = e.what();
        return int(e.status);
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return DQ_MEMORY_ERROR;
    } catch (const std::exception& e) {
        g_error = e.what();
        return DQ_RUNTIME_ERROR;
    } catch (...) {
        g_error = "unknown error";
        return DQ_RUNTIME_ERROR;
    }
}

void need(const void* p, const char* what) {
    if (!p) fail(kValueError, std::string("null pointer: ") + what);
}

std::vector<uint64_t> query_qubits(const dq_result* r, const uint64_t* qubits, size_t k, int has) {
    std::vector<uint64_t> q;
    uint64_t n = r->impl->n;
    if (!has) {
        for (uint64_t i = 0; i < n; i++) q.push_back(n - 1 - i);
        return q;
    }
    // validate_query, simulator.rs:193-202
    for (size_t i = 0; i < k; i++) {
        bool dup = false;
        for (size_t j = 0; j < i; j++) dup = dup || qubits[j] == qubits[i];
        if (qubits[i] >= n || dup) fail(kValueError, "Query qubits must be distinct and within the statevector's range");
        q.push_back(qubits[i]);
    }
    return q;
}
}  // namespace

extern "C" {

const char* dq_last_error(void) { return g_error.c_str(); }

const char* dq_version(void) { return "dqsim-b200 0.1.2"; }

void dq_sim_options_default(dq_sim_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_memory_mb = 1024;
    o->sample_terminal = 1;
    o->precision = DQ_COMPLEX128;
}

int dq_sim_create(const dq_sim_options* opts, dq_sim** out) {
    return guard([&] {
        need(opts, "opts");
        need(out, "out");
        Options o;
        o.has_seed = opts->has_seed != 0;
        o.seed = opts->seed;
        o.profile = opts->profile != 0;
        o.max_memory_mb = opts->max_memory_mb;
        o.has_max_parallel_shots = opts->has_max_parallel_shots != 0;
        o.max_parallel_shots = opts->max_parallel_shots;
        o.sample_terminal = opts->sample_terminal != 0;
        if (opts->precision != DQ_COMPLEX128 && opts->precision != DQ_COMPLEX64)
            fail(kValueError, "precision must be complex128 or complex64");
        o.precision = Precision(opts->precision);
        o.device = opts->device;
        if (opts->execution < 0 || opts->execution > 2) fail(kValueError, "execution must be auto, per_gate or tiled");
        if (opts->tile_qubits < 0 || opts->tile_qubits > 14 || (opts->tile_qubits > 0 && opts->tile_qubits < 5))
            fail(kValueError, "tile_qubits must be 0 (auto) or between 5 and 14");
        if (opts->tile_qubits == 14 && opts->precision == DQ_COMPLEX128)
            fail(kValueError, "a 14-qubit complex128 tile exceeds shared memory");
        if (opts->fusion_width < 0 || opts->fusion_width > 5) fail(kValueError, "fusion_width must be between 0 and 5");
        o.execution = opts->execution;
        o.tile_qubits = opts->tile_qubits;
        o.fusion_width = opts->fusion_width;
        auto s = std::make_unique<dq_sim>();
        s->impl = std::make_unique<Simulator>(o);
        *out = s.release();
    });
}

void dq_sim_destroy(dq_sim* sim) { delete sim; }

int dq_simulate_shots(dq_sim* sim, const char* json, size_t len, uint64_t shots, int profile, dq_counts** out) {
    return guard([&] {
        need(sim, "sim");
        need(json, "json");
        need(out, "out");
        ShotOutput so = sim->impl->simulate_shots(json, len, shots, profile != 0, nullptr, nullptr);
        auto c = std::make_unique<dq_counts>();
        if (!so.flat_counts.empty()) {
            c->width = so.key_width;
            c->keys = std::move(so.flat_keys);
            c->counts = std::move(so.flat_counts);
        } else {
            for (auto& kv : so.counts) {
                c->width = kv.first.size();
                c->keys += kv.first;
                c->counts.push_back(kv.second);
            }
        }
        *out = c.release();
    });
}

int dq_simulate(dq_sim* sim, const char* json, size_t len, dq_result** out) {
    return guard([&] {
        need(sim, "sim");
        need(json, "json");
        need(out, "out");
        auto r = std::make_unique<dq_result>();
        r->impl = sim->impl->simulate(json, len);
        *out = r.release();
    });
}

int dq_counts_size(const dq_counts* c, uint64_t* n_keys, uint64_t* key_width) {
    return guard([&] {
        need(c, "counts");
        if (n_keys) *n_keys = c->counts.size();
        if (key_width) *key_width = c->width;
    });
}

int dq_counts_copy(const dq_counts* c, char* keys, uint64_t* counts) {
    return guard([&] {
        need(c, "counts");
        if (keys && !c->keys.empty()) std::memcpy(keys, c->keys.data(), c->keys.size());
        if (counts && !c->counts.empty()) std::memcpy(counts, c->counts.data(), c->counts.size() * 8);
    });
}

void dq_counts_free(dq_counts* c) { delete c; }

int dq_result_num_qubits(const dq_result* r, uint64_t* n) {
    return guard([&] {
        need(r, "result");
        need(n, "n");
        *n = r->impl->n;
    });
}

int dq_result_num_cbits(const dq_result* r, uint64_t* n) {
    return guard([&] {
        need(r, "result");
        need(n, "n");
        *n = r->impl->cbits.size();
    });
}

int dq_result_statevector(const dq_result* r, double* out, uint64_t out_len) {
    return guard([&] {
        need(r, "result");
        need(out, "out");
        if (out_len != (uint64_t(2) << r->impl->n)) fail(kValueError, "statevector buffer has the wrong length");
        r->impl->statevector(out);
    });
}

int dq_result_classical_bits(const dq_result* r, uint8_t* out, uint64_t out_len) {
    return guard([&] {
        need(r, "result");
        if (out_len != r->impl->cbits.size()) fail(kValueError, "classical bit buffer has the wrong length");
        if (out_len) std::memcpy(out, r->impl->cbits.data(), out_len);
    });
}

int dq_result_profile(const dq_result* r, dq_profile* out, int* has) {
    return guard([&] {
        need(r, "result");
        need(out, "out");
        need(has, "has");
        const ProfileData& p = r->impl->profile;
        *has = p.present ? 1 : 0;
        out->apply_one_qubit_calls = p.acc.oq_calls;
        out->apply_one_qubit_time = p.acc.oq_time;
        out->apply_n_qubit_calls = p.acc.nq_calls;
        out->apply_n_qubit_time = p.acc.nq_time;
        out->measure_qubit_calls = p.acc.mq_calls;
        out->measure_qubit_time = p.acc.mq_time;
        out->total_time = p.total_time;
    });
}

int dq_result_probabilities(const dq_result* r, const uint64_t* qubits, size_t k, int has_qubits, double* out,
                            uint64_t out_len) {
    return guard([&] {
        need(r, "result");
        auto q = query_qubits(r, qubits, k, has_qubits);
        if (out_len != (uint64_t(1) << q.size())) fail(kValueError, "probability buffer has the wrong length");
        need(out, "out");
        r->impl->probabilities(q, out);
    });
}

int dq_result_counts(const dq_result* r, uint64_t shots, const uint64_t* qubits, size_t k, int has_qubits,
                     uint64_t seed, int has_seed, dq_counts** out) {
    return guard([&] {
        need(r, "result");
        need(out, "out");
        auto q = query_qubits(r, qubits, k, has_qubits);
        if (!has_seed) {
            std::random_device rd;
            seed = (uint64_t(rd()) << 32) ^ uint64_t(rd());
        }
        auto m = r->impl->counts(shots, q, seed);
        auto c = std::make_unique<dq_counts>();
        c->width = q.size();
        for (auto& kv : m) {
            std::string key(q.size(), '0');
            for (size_t b = 0; b < q.size(); b++)
                if ((kv.first >> (q.size() - 1 - b)) & 1) key[b] = '1';
            c->keys += key;
            c->counts.push_back(kv.second);
        }
        *out = c.release();
    });
}

int dq_result_amplitudes(const dq_result* r, const uint64_t* indices, uint64_t count, double* out) {
    return guard([&] {
        need(r, "result");
        if (count) {
            need(indices, "indices");
            need(out, "out");
        }
        r->impl->amplitudes(indices, count, out);
    });
}

int dq_debug_fused_fault(uint64_t withhold_step, double wait_ms) {
    return guard([&] { k::set_fused_fault(withhold_step, wait_ms); });
}

int dq_result_pauli_expectation(const dq_result* r, uint64_t x_mask, uint64_t z_mask, double* re, double* im) {
    return guard([&] {
        need(r, "result");
        need(re, "re");
        need(im, "im");
        r->impl->pauli_xz(x_mask, z_mask, re, im);
        // X^x Z^z differs from the Pauli product by i per Y (Y = i X Z).
        const int ny = __builtin_popcountll(x_mask & z_mask) & 3;
        for (int k = 0; k < ny; k++) {
            const double t = *re;
            *re = -*im;
            *im = t;
        }
    });
}

int dq_result_fidelity(const dq_result* r, const double* other, uint64_t other_len, double* out) {
    return guard([&] {
        need(r, "result");
        need(out, "out");
        if (other_len != (uint64_t(1) << r->impl->n)) {
            *out = 0.0;
            return;
        }
        need(other, "other");
        *out = r->impl->fidelity(other, other_len);
    });
}

void dq_result_free(dq_result* r) { delete r; }

int dq_plan_create(dq_sim* sim, const char* json, size_t len, uint64_t shots, dq_plan** out) {
    return guard([&] {
        need(sim, "sim");
        need(json, "json");
        need(out, "out");
        auto p = std::make_unique<dq_plan>();
        p->impl = std::make_unique<Plan>(*sim->impl, json, len, shots);
        *out = p.release();
    });
}

int dq_plan_run(dq_plan* p, int record, double* device_ms) {
    return guard([&] {
        need(p, "plan");
        double ms = p->impl->run(record != 0);
        if (device_ms) *device_ms = ms;
    });
}

int dq_plan_stats(const dq_plan* p, double* ms, uint64_t* launches, double* bytes) {
    return guard([&] {
        need(p, "plan");
        need(ms, "ms");
        need(launches, "launches");
        need(bytes, "bytes");
        p->impl->stats(ms, launches, bytes);
    });
}

int dq_plan_info(const dq_plan* p, uint64_t* num_qubits, uint64_t* num_ops, double* state_bytes) {
    return guard([&] {
        need(p, "plan");
        if (num_qubits) *num_qubits = p->impl->num_qubits();
        if (num_ops) *num_ops = p->impl->num_ops();
        if (state_bytes) *state_bytes = p->impl->state_bytes();
    });
}

int dq_plan_statevector(const dq_plan* p, double* out, uint64_t out_len) {
    return guard([&] {
        need(p, "plan");
        need(out, "out");
        if (out_len != (uint64_t(2) << p->impl->num_qubits())) fail(kValueError, "statevector buffer has the wrong length");
        p->impl->statevector(out);
    });
}

int dq_plan_samples(const dq_plan* p, uint64_t* out, uint64_t out_len) {
    return guard([&] {
        need(p, "plan");
        need(out, "out");
        if (out_len != p->impl->shots()) fail(kValueError, "sample buffer has the wrong length");
        p->impl->samples(out);
    });
}

int dq_plan_compare(const dq_plan* a, const dq_plan* b, double* fidelity, double* max_abs_err) {
    return guard([&] {
        need(a, "a");
        need(b, "b");
        need(fidelity, "fidelity");
        need(max_abs_err, "max_abs_err");
        a->impl->compare(*b->impl, fidelity, max_abs_err);
    });
}

void dq_plan_free(dq_plan* p) { delete p; }

int dq_batch_create(dq_sim* sim, const char* const* jsons, const size_t* lens, uint64_t count, uint64_t shots,
                    int autotune, dq_batch** out) {
    return guard([&] {
        need(sim, "sim");
        need(out, "out");
        if (count == 0) fail(kValueError, "a batch needs at least one circuit");
        need(jsons, "jsons");
        need(lens, "json_lens");
        std::vector<std::string> texts;
        for (uint64_t i = 0; i < count; i++) {
            need(jsons[i], "json");
            texts.emplace_back(jsons[i], lens[i]);
        }
        BatchTuning t;
        if (autotune < 0 || autotune > 2) fail(kValueError, "autotune must be 0, 1 or 2");
        if (autotune == 2) t.fuse = 5;  // tensor-core fused passes wherever they apply
        if (autotune == 1) {
            const bool c64 = sim->impl->options().precision == Precision::C64;
            std::map<uint64_t, size_t> first;
            for (size_t i = 0; i < texts.size(); i++) {
                uint64_t n = 0;
                compile_json(texts[i].data(), texts[i].size(), &n, nullptr);
                first.emplace(n, i);
            }
            for (auto& kv : first) {
                TuneResult r = autotune_tile(*sim->impl, texts[kv.second], c64);
                t.per_n[kv.first] = BatchShape{r.tile_m, r.fuse, r.depth};
            }
        }
        auto b = std::make_unique<dq_batch>();
        b->impl = std::make_unique<BatchRun>(*sim->impl, texts, shots, t);
        *out = b.release();
    });
}

int dq_batch_run(dq_batch* b, int use_graph, double* device_ms) {
    return guard([&] {
        need(b, "batch");
        double ms = b->impl->run(use_graph != 0);
        if (device_ms) *device_ms = ms;
    });
}

int dq_batch_counts(const dq_batch* b, uint64_t index, dq_counts** out) {
    return guard([&] {
        need(b, "batch");
        need(out, "out");
        if (index >= b->impl->size()) fail(kValueError, "batch index out of range");
        auto m = b->impl->counts(size_t(index));
        auto c = std::make_unique<dq_counts>();
        for (auto& kv : m) {
            c->width = kv.first.size();
            c->keys += kv.first;
            c->counts.push_back(kv.second);
        }
        *out = c.release();
    });
}

int dq_batch_expect_zz(const dq_batch* b, double* out, uint64_t count) {
    return guard([&] {
        need(b, "batch");
        need(out, "out");
        if (count != b->impl->size()) fail(kValueError, "expectation buffer has the wrong length");
        auto v = b->impl->expect_zz();
        std::copy(v.begin(), v.end(), out);
    });
}

int dq_batch_statevector(const dq_batch* b, uint64_t index, double* out, uint64_t out_len) {
    return guard([&] {
        need(b, "batch");
        need(out, "out");
        if (index >= b->impl->size()) fail(kValueError, "batch index out of range");
        if (out_len != (uint64_t(2) << b->impl->num_qubits(size_t(index))))
            fail(kValueError, "statevector buffer has the wrong length");
        b->impl->statevector(size_t(index), out);
    });
}

int dq_batch_info(const dq_batch* b, uint64_t* passes, uint64_t* items) {
    return guard([&] {
        need(b, "batch");
        if (passes) *passes = b->impl->passes();
        if (items) *items = b->impl->items();
    });
}

int dq_batch_work(const dq_batch* b, double* bytes, double* tensor_flops, double* cuda_core_flops,
                  uint64_t* fused_circuits) {
    return guard([&] {
        need(b, "batch");
        double by = 0, tf = 0, cf = 0;
        b->impl->work(&by, &tf, &cf);
        if (bytes) *bytes = by;
        if (tensor_flops) *tensor_flops = tf;
        if (cuda_core_flops) *cuda_core_flops = cf;
        if (fused_circuits) *fused_circuits = b->impl->fused_circuits();
    });
}

void dq_batch_free(dq_batch* b) { delete b; }

int dq_cost_model_create(int device, uint64_t seed, dq_cost_model** out) {
    return dq_cost_model_create_kind(device, seed, DQ_COST_TILE_OPS, out);
}

int dq_cost_model_create_kind(int device, uint64_t seed, int kind, dq_cost_model** out) {
    return guard([&] {
        need(out, "out");
        auto m = std::make_unique<dq_cost_model>();
        m->impl = std::make_unique<CostModel>(device, seed, kind);
        *out = m.release();
    });
}

int dq_cost_model_kind(const dq_cost_model* m, int* kind) {
    return guard([&] {
        need(m, "model");
        need(kind, "kind");
        *kind = m->impl->kind();
    });
}

namespace {
void give_text(const std::string& s, char** out_text) {
    char* buf = static_cast<char*>(std::malloc(s.size() + 1));
    if (!buf) throw std::bad_alloc();
    std::memcpy(buf, s.c_str(), s.size() + 1);
    *out_text = buf;
}
}  // namespace

int dq_fused_portfolio(dq_sim* sim, const char* json, size_t len, int wide, int measure, const dq_cost_model* model,
                       char** out_text) {
    return guard([&] {
        need(sim, "sim");
        need(json, "json");
        need(out_text, "out_text");
        give_text(fused_portfolio_json(*sim->impl, json, len, wide != 0, measure != 0, model ? model->impl.get() : nullptr),
                  out_text);
    });
}

int dq_fused_pass_features(int num_qubits, const int* tile_qubits, int nblocks, int gates, float* out) {
    return guard([&] {
        need(tile_qubits, "tile_qubits");
        need(out, "out");
        if (num_qubits < kFusedM || num_qubits > 63) fail(kValueError, "num_qubits must be between 12 and 63");
        std::vector<int> tq(tile_qubits, tile_qubits + kFusedM);
        for (size_t i = 0; i < tq.size(); i++)
            if (tq[i] < 0 || tq[i] >= num_qubits || (i && tq[i] <= tq[i - 1]))
                fail(kValueError, "tile qubits must be 12 ascending qubits of the state");
        fused_pass_features(num_qubits, 1, tq, nblocks, gates, out);
    });
}

int dq_fused_random_passes(dq_sim* sim, int num_qubits, uint64_t count, uint64_t seed, int measure, char** out_text) {
    return guard([&] {
        need(sim, "sim");
        need(out_text, "out_text");
        give_text(fused_random_passes_json(*sim->impl, num_qubits, count, seed, measure != 0), out_text);
    });
}

void dq_cost_model_free(dq_cost_model* m) { delete m; }

int dq_cost_model_add_samples(dq_cost_model* m, const float* features, const float* log_cycles, uint64_t n) {
    return guard([&] {
        need(m, "model");
        if (n) {
            need(features, "features");
            need(log_cycles, "log_cycles");
        }
        m->impl->add_samples(features, log_cycles, size_t(n));
    });
}

int dq_cost_model_record(dq_cost_model* m, dq_sim* sim, const char* json, size_t len, uint64_t* added) {
    return guard([&] {
        need(m, "model");
        need(sim, "sim");
        need(json, "json");
        Plan p(*sim->impl, json, len, 0);
        std::vector<float> X, y;
        p.record_costs(X, y);
        m->impl->add_samples(X.data(), y.data(), y.size());
        if (added) *added = y.size();
    });
}

int dq_cost_model_num_samples(const dq_cost_model* m, uint64_t* n) {
    return guard([&] {
        need(m, "model");
        need(n, "n");
        *n = m->impl->num_samples();
    });
}

int dq_cost_model_samples(const dq_cost_model* m, float* features, float* log_cycles, uint64_t n) {
    return guard([&] {
        need(m, "model");
        if (n != m->impl->num_samples()) fail(kValueError, "sample buffers have the wrong length");
        m->impl->copy_samples(features, log_cycles);
    });
}

int dq_cost_model_train(dq_cost_model* m, int epochs, float lr, double* final_mse) {
    return guard([&] {
        need(m, "model");
        if (epochs < 1 || !(lr > 0.f)) fail(kValueError, "epochs must be positive and lr > 0");
        double l = m->impl->train(epochs, lr);
        if (final_mse) *final_mse = l;
    });
}

int dq_cost_model_predict(const dq_cost_model* m, const float* features, uint64_t n, float* log_cycles) {
    return guard([&] {
        need(m, "model");
        if (n) {
            need(features, "features");
            need(log_cycles, "log_cycles");
        }
        m->impl->predict(features, size_t(n), log_cycles);
    });
}

int dq_cost_model_gradients(const dq_cost_model* m, const float* features, const float* log_cycles, uint64_t n,
                            float* grads) {
    return guard([&] {
        need(m, "model");
        need(features, "features");
        need(log_cycles, "log_cycles");
        need(grads, "grads");
        m->impl->gradients(features, log_cycles, size_t(n), grads);
    });
}

int dq_cost_model_get_params(const dq_cost_model* m, float* out, uint64_t len) {
    return guard([&] {
        need(m, "model");
        need(out, "out");
        if (len != uint64_t(kMlpParams + 2)) fail(kValueError, "parameter buffer must hold DQ_MLP_PARAMS floats");
        m->impl->get_params(out);
    });
}

int dq_cost_model_set_params(dq_cost_model* m, const float* in, uint64_t len) {
    return guard([&] {
        need(m, "model");
        need(in, "in");
        if (len != uint64_t(kMlpParams + 2)) fail(kValueError, "parameter buffer must hold DQ_MLP_PARAMS floats");
        m->impl->set_params(in);
    });
}

int dq_sim_set_cost_model(dq_sim* sim, dq_cost_model* m) {
    return guard([&] {
        need(sim, "sim");
        if (m && !m->impl->trained()) fail(kValueError, "attach a trained cost model");
        sim->impl->set_cost_model(m ? m->impl.get() : nullptr);
    });
}

int dq_plan_planner(const dq_plan* p, double* learned_ms, double* greedy_ms, int* used_learned, int* rejected) {
    return guard([&] {
        need(p, "plan");
        double a, b;
        int u, r;
        p->impl->planner(&a, &b, &u, &r);
        if (learned_ms) *learned_ms = a;
        if (greedy_ms) *greedy_ms = b;
        if (used_learned) *used_learned = u;
        if (rejected) *rejected = r;
    });
}

int dq_plan_flops(const dq_plan* p, double* cuda_core_flops, double* tensor_flops) {
    return guard([&] {
        need(p, "plan");
        need(cuda_core_flops, "cuda_core_flops");
        need(tensor_flops, "tensor_flops");
        p->impl->flops(cuda_core_flops, tensor_flops);
    });
}

int dq_plan_shape(const dq_plan* p, uint64_t* passes, uint64_t* tile_ops, uint64_t* fused_blocks) {
    return guard([&] {
        need(p, "plan");
        if (passes) *passes = p->impl->passes();
        if (tile_ops) *tile_ops = p->impl->tile_ops();
        if (fused_blocks) *fused_blocks = p->impl->fused_blocks();
    });
}

int dq_sim_planner_log(dq_sim* sim, char** out_text) {
    return guard([&] {
        need(sim, "sim");
        need(out_text, "out_text");
        std::string s = sim->impl->planner_log();
        char* buf = static_cast<char*>(std::malloc(s.size() + 1));
        if (!buf) throw std::bad_alloc();
        std::memcpy(buf, s.c_str(), s.size() + 1);
        *out_text = buf;
    });
}

int dq_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes) {
    return guard([&] {
        need(free_bytes, "free_bytes");
        need(total_bytes, "total_bytes");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
            cudaGetLastError();
            fail(kValueError, "CUDA device ordinal out of range");
        }
        int prev = 0;
        cudaGetDevice(&prev);
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        size_t f = 0, tot = 0;
        const cudaError_t e = cudaMemGetInfo(&f, &tot);
        cudaSetDevice(prev);
        cuda_check(e, "cudaMemGetInfo");
        *free_bytes = f;
        *total_bytes = tot;
    });
}

int dq_device_fp64_tflops(int device, double* tflops) {
    return guard([&] {
        need(tflops, "tflops");
        *tflops = fp64_fma_tflops(device);
    });
}

int dq_sim_last_call_phases(dq_sim* sim, double* out, uint64_t n) {
    return guard([&] {
        need(sim, "sim");
        need(out, "out");
        if (n != uint64_t(kNumCallPhases)) fail(kValueError, "phase buffer must hold DQ_CALL_PHASES doubles");
        sim->impl->last_call_phases(out);
    });
}

int dq_measure_noalloc(void* states, int precision, uint64_t num_states, uint64_t num_qubits, uint64_t qubit,
                       int reset, const uint64_t* seeds, const uint64_t* draw_index, int* outcomes) {
    return guard([&] {
        measure_noalloc(states, precision, num_states, num_qubits, qubit, reset, seeds, draw_index, outcomes);
    });
}

int dq_blocks_create(int device, int precision, dq_blocks** out) {
    return guard([&] {
        need(out, "out");
        if (precision != DQ_COMPLEX128 && precision != DQ_COMPLEX64)
            fail(kValueError, "precision must be DQ_COMPLEX128 or DQ_COMPLEX64");
        auto b = std::make_unique<dq_blocks>();
        b->impl = std::make_unique<BlockContext>(device, precision == DQ_COMPLEX64);
        *out = b.release();
    });
}

void dq_blocks_destroy(dq_blocks* ctx) { delete ctx; }

int dq_blocks_sync(dq_blocks* ctx) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->sync();
    });
}

int dq_block_apply_one_qubit(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t target, const double* matrix,
                             const uint64_t* ctl_qubits, const uint8_t* ctl_values, size_t num_controls) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->apply_one_qubit(state, num_qubits, target, matrix, ctl_qubits, ctl_values, num_controls, false);
    });
}

int dq_block_apply_x(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t target, const uint64_t* ctl_qubits,
                     const uint8_t* ctl_values, size_t num_controls) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->apply_one_qubit(state, num_qubits, target, nullptr, ctl_qubits, ctl_values, num_controls, true);
    });
}

int dq_block_apply_swap(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t a, uint64_t b,
                        const uint64_t* ctl_qubits, const uint8_t* ctl_values, size_t num_controls) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->apply_swap(state, num_qubits, a, b, ctl_qubits, ctl_values, num_controls);
    });
}

int dq_block_apply_diagonal(dq_blocks* ctx, void* state, uint64_t num_qubits, const uint64_t* qubits, size_t k,
                            const double* diagonal) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->apply_diagonal(state, num_qubits, qubits, k, diagonal);
    });
}

int dq_block_apply_dense(dq_blocks* ctx, void* state, uint64_t num_qubits, const uint64_t* qubits, size_t k,
                         const double* matrix) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->apply_dense(state, num_qubits, qubits, k, matrix);
    });
}

int dq_block_measure(dq_blocks* ctx, void* state, uint64_t num_qubits, uint64_t qubit, double draw, int* outcome) {
    return guard([&] {
        need(ctx, "ctx");
        need(outcome, "outcome");
        *outcome = ctx->impl->measure(state, num_qubits, qubit, draw);
    });
}

int dq_block_merge(dq_blocks* ctx, const void* left, uint64_t left_qubits, const void* right, uint64_t right_qubits,
                   void* out) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->merge(left, left_qubits, right, right_qubits, out);
    });
}

int dq_block_probabilities(dq_blocks* ctx, const void* state, uint64_t num_qubits, const uint64_t* qubits, size_t k,
                           double* out) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->probabilities(state, num_qubits, qubits, k, out);
    });
}

int dq_block_running_sums(dq_blocks* ctx, const void* state, uint64_t num_qubits, double* out) {
    return guard([&] {
        need(ctx, "ctx");
        ctx->impl->running_sums(state, num_qubits, out);
    });
}

int dq_compile_dump(const char* json, size_t len, char** out_text) {
    return guard([&] {
        need(json, "json");
        need(out_text, "out_text");
        auto ops = compile_json(json, len, nullptr, nullptr);
        std::string s = dump_operations(ops);
        char* buf = static_cast<char*>(std::malloc(s.size() + 1));
        if (!buf) throw std::bad_alloc();
        std::memcpy(buf, s.c_str(), s.size() + 1);
        *out_text = buf;
    });
}

int dq_tile_plan_dump(const char* json, size_t len, int tile_qubits, int fusion_width, char** out_text) {
    return guard([&] {
        need(json, "json");
        need(out_text, "out_text");
        uint64_t n = 0, ncb = 0;
        auto ops = compile_json(json, len, &n, &ncb);
        for (auto& op : ops)
            if (!tileable(op)) fail(kValueError, "circuit has operations a tile pass cannot apply");
        TilePlanOptions o;
        o.m = tile_qubits;
        o.fuse = std::min(fusion_width, kTileMaxDense);
        o.beam = kPlanBeam;
        std::vector<double2> pool;
        auto passes = plan_tiles(ops, 0, ops.size(), int(n), o, &pool);
        std::string s = "{\"n\":" + std::to_string(n) + ",\"passes\":[";
        char buf[64];
        for (size_t pi = 0; pi < passes.size(); pi++) {
            const TilePass& p = passes[pi];
            s += pi ? ",{" : "{";
            s += "\"raw\":" + std::to_string(p.raw_ops) + ",\"qubits\":[";
            for (size_t i = 0; i < p.qubits.size(); i++) s += (i ? "," : "") + std::to_string(p.qubits[i]);
            s += "],\"ops\":[";
            for (size_t oi = 0; oi < p.ops.size(); oi++) {
                const TileOp& t = p.ops[oi];
                s += oi ? ",{" : "{";
                s += "\"type\":" + std::to_string(t.type) + ",\"k\":" + std::to_string(t.k) + ",\"ins\":[";
                for (int i = 0; i < t.nins; i++) s += (i ? "," : "") + std::to_string(t.ins[i]);
                s += "],\"q\":[";
                for (int i = 0; i < t.k; i++) s += (i ? "," : "") + std::to_string(t.q[i]);
                s += "],\"offs\":[";
                for (int i = 0; t.type == TileOp::kDense && i < (1 << t.k); i++)
                    s += (i ? "," : "") + std::to_string(t.offs[i]);
                s += "],\"fixed\":" + std::to_string(t.fixed) + ",\"tbit\":" + std::to_string(t.tbit) +
                     ",\"lowbit\":" + std::to_string(t.lowbit) + ",\"highbit\":" + std::to_string(t.highbit) +
                     ",\"mat\":" + std::to_string(t.mat) + "}";
            }
            // The pass's register phases (complex128 swizzle), decoded from the
            // block the executor plans: offsets of every register entry and slot
            // bit, and each operation with its matrix appended to the pool.
            s += "],\"phases\":[";
            if (phase_supported(int(p.qubits.size()))) {
                std::vector<uint4> blk;
                const int nph = plan_phases(p.ops, int(p.qubits.size()), false, pool, blk);
                auto arr = [](const std::vector<uint32_t>& v) {
                    std::string a = "[";
                    for (size_t i = 0; i < v.size(); i++) a += (i ? "," : "") + std::to_string(v[i]);
                    return a + "]";
                };
                for (int hi = 0; hi < nph; hi++) {
                    const uint4* h = &blk[size_t(hi) * kPhaseWords];
                    const uint32_t rp[4] = {h[1].x, h[1].y, h[1].z, h[1].w};
                    std::vector<uint32_t> rb, prb, sb, psb;
                    for (int v = 0; v < kPhaseEntries; v++) {
                        uint32_t o = 0, po = 0;
                        for (int i = 0; i < kPhaseRegBits; i++)
                            if ((v >> i) & 1) {
                                o |= rp[i] & 0xFFFFu;
                                po ^= rp[i] >> 16;
                            }
                        rb.push_back(o);
                        prb.push_back(po);
                    }
                    for (uint32_t i = 0; i < h[0].z; i++) {
                        const uint4 w = h[2 + i / 4];
                        const uint32_t sp = (i % 4 == 0 ? w.x : i % 4 == 1 ? w.y : i % 4 == 2 ? w.z : w.w);
                        sb.push_back(sp & 0xFFFFu);
                        psb.push_back(sp >> 16);
                    }
                    s += hi ? ",{" : "{";
                    s += "\"rb\":" + arr(rb) + ",\"prb\":" + arr(prb) + ",\"sb\":" + arr(sb) + ",\"psb\":" +
                         arr(psb) + ",\"ops\":[";
                    for (uint32_t oi = 0; oi < h[0].y; oi++) {
                        const uint4 o0 = blk[h[0].x + kPhaseOpWords * oi], o1 = blk[h[0].x + kPhaseOpWords * oi + 1];
                        const int code = int(o0.x), k = int(o1.x);
                        int count = 0;  // matrix words of the operation
                        if (code < kPhX || code == kPhOne + 3) count = 4;
                        else if (code >= kPhD2 && code < kPhD3) count = 16;
                        else if (code >= kPhD3 && code < kPhSwap) count = 64;
                        else if (code == kPhDiagEntry) count = 1;
                        else if (code == kPhDiagFull) count = 1 << k;
                        const size_t mat = pool.size();
                        for (int e = 0; e < count; e++) {
                            double2 v;
                            std::memcpy(&v, &blk[o0.y + uint32_t(e)], sizeof v);
                            pool.push_back(v);
                        }
                        s += oi ? ",{" : "{";
                        s += "\"code\":" + std::to_string(code) + ",\"mat\":" + std::to_string(mat) +
                             ",\"mask\":" + std::to_string(o0.z) + ",\"value\":" + std::to_string(o0.w) +
                             ",\"k\":" + std::to_string(k) + ",\"q\":[";
                        for (int b = 0; b < k; b++)
                            s += (b ? "," : "") + std::to_string(((b < 4 ? o1.y : o1.z) >> (8 * (b & 3))) & 0xFFu);
                        s += "]}";
                    }
                    s += "]}";
                }
            }
            s += "]}";
        }
        s += "],\"pool\":[";
        for (size_t i = 0; i < pool.size(); i++) {
            std::snprintf(buf, sizeof buf, "%s[%.17g,%.17g]", i ? "," : "", pool[i].x, pool[i].y);
            s += buf;
        }
        s += "]}";
        char* out = static_cast<char*>(std::malloc(s.size() + 1));
        if (!out) throw std::bad_alloc();
        std::memcpy(out, s.c_str(), s.size() + 1);
        *out_text = out;
    });
}

int dq_fused_plan_dump(const char* json, size_t len, char** out_text) {
    return guard([&] {
        need(json, "json");
        need(out_text, "out_text");
        uint64_t n = 0, ncb = 0;
        auto ops = compile_json(json, len, &n, &ncb);
        for (auto& op : ops)
            if (!op.is_unitary()) fail(kValueError, "circuit has non-unitary operations");
        if (n < uint64_t(kFusedM)) fail(kValueError, "fused passes need at least 12 qubits");
        // The simulator's own plan (plan_fused), its passes' blocks and gate
        // images concatenated in pass order.
        std::vector<BuiltFusedPass> passes = plan_fused(ops, 0, ops.size(), int(n), TilePlanOptions{});
        std::vector<FusedBlock> blocks;
        std::vector<uint16_t> upool;
        std::string s = "{\"n\":" + std::to_string(n) + ",\"passes\":[";
        char buf[48];
        for (size_t pi = 0; pi < passes.size(); pi++) {
            FusedPass fp = passes[pi].fp;
            fp.first_block += int(blocks.size());
            for (FusedBlock b : passes[pi].blocks) {
                b.u_off += uint32_t(upool.size());
                blocks.push_back(b);
            }
            upool.insert(upool.end(), passes[pi].upool.begin(), passes[pi].upool.end());
            s += pi ? ",{" : "{";
            s += "\"raw\":" + std::to_string(fp.raw_ops) + ",\"qubits\":[";
            for (size_t i = 0; i < fp.qubits.size(); i++) s += (i ? "," : "") + std::to_string(fp.qubits[i]);
            s += "],\"in_lo\":[";
            for (int i = 0; i < 64; i++) s += (i ? "," : "") + std::to_string(fp.in_lo[i]);
            s += "],\"in_hi\":[";
            for (int i = 0; i < 64; i++) s += (i ? "," : "") + std::to_string(fp.in_hi[i]);
            s += "],\"out_lo\":[";
            for (int i = 0; i < 64; i++) s += (i ? "," : "") + std::to_string(fp.out_lo[i]);
            s += "],\"out_hi\":[";
            for (int i = 0; i < 64; i++) s += (i ? "," : "") + std::to_string(fp.out_hi[i]);
            s += "],\"split_pos\":[";
            for (int i = 0; i < 8; i++) s += (i ? "," : "") + std::to_string(fp.split_pos[i]);
            s += "],\"split_q\":[";
            for (int i = 0; i < 16; i++) s += (i ? "," : "") + std::to_string(fp.split_q[i]);
            s += "],\"split_qoff\":[";
            for (int i = 0; i < 16; i++) s += (i ? "," : "") + std::to_string(fp.split_qoff[i]);
            const FusedTma t = fused_tma_plan(fp.qubits, int(n), 1);
            s += "],\"tma\":{\"ok\":" + std::to_string(t.ok) + ",\"dims\":" + std::to_string(t.dims) +
                 ",\"copies\":" + std::to_string(t.copies) + ",\"copy_bytes\":" + std::to_string(t.copy_bytes);
            const char* names[4] = {"lo", "bits", "box", "extent"};
            for (int f = 0; f < 4; f++) {
                s += std::string(",\"") + names[f] + "\":[";
                for (int i = 0; i < 5; i++) {
                    const uint64_t v = f == 0 ? uint64_t(t.lo[i]) : f == 1 ? uint64_t(t.bits[i]) : f == 2 ? t.box[i] : t.extent[i];
                    s += (i ? "," : "") + std::to_string(v);
                }
                s += "]";
            }
            s += ",\"copy_step\":[";
            for (int c = 0; c < t.copies; c++) s += (c ? "," : "") + std::to_string(t.copy_step[c]);
            s += "]},\"blocks\":[";
            for (int bi = 0; bi < fp.nblocks; bi++) {
                const FusedBlock& b = blocks[size_t(fp.first_block + bi)];
                s += bi ? ",{" : "{";
                s += "\"u_off\":" + std::to_string(b.u_off) + ",\"last\":" + std::to_string(b.last) + ",\"mask\":" +
                     std::to_string(size_t(bi) < fp.block_masks.size() ? fp.block_masks[size_t(bi)] : 0u) +
                     ",\"next_b\":[";
                for (int i = 0; i < 32; i++) s += (i ? "," : "") + std::to_string(b.next_b[i]);
                s += "],\"next_c\":[";
                for (int i = 0; i < kFusedCols; i++) s += (i ? "," : "") + std::to_string(b.next_c[i]);
                s += "]}";
            }
            s += "]}";
        }
        s += "],\"upool\":[";
        for (size_t i = 0; i < upool.size(); i++) {
            std::snprintf(buf, sizeof buf, "%s%u", i ? "," : "", unsigned(upool[i]));
            s += buf;
        }
        s += "]}";
        char* outp = static_cast<char*>(std::malloc(s.size() + 1));
        if (!outp) throw std::bad_alloc();
        std::memcpy(outp, s.c_str(), s.size() + 1);
        *out_text = outp;
    });
}

void dq_string_free(char* s) { std::free(s); }

}  // extern "C"

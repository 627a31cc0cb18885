// extern "C" layer: exceptions become status codes plus a thread-local message.
#include <cstdlib>
#include <cstring>
#include <random>

#include "../../include/dqsim_sv.h"
#include "simulator.hpp"

using namespace dq;

struct dq_sim {
    std::unique_ptr<Simulator> impl;
};
struct dq_result {
    std::unique_ptr<Result> impl;
};
struct dq_counts {
    uint64_t width = 0;
    std::vector<std::string> keys;
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
        c->width = 0;
        for (auto& kv : so.counts) {
            c->width = kv.first.size();
            c->keys.push_back(kv.first);
            c->counts.push_back(kv.second);
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
        if (n_keys) *n_keys = c->keys.size();
        if (key_width) *key_width = c->width;
    });
}

int dq_counts_copy(const dq_counts* c, char* keys, uint64_t* counts) {
    return guard([&] {
        need(c, "counts");
        for (size_t i = 0; i < c->keys.size(); i++) {
            if (keys && c->width) std::memcpy(keys + i * c->width, c->keys[i].data(), c->width);
            if (counts) counts[i] = c->counts[i];
        }
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
            c->keys.push_back(key);
            c->counts.push_back(kv.second);
        }
        *out = c.release();
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

void dq_string_free(char* s) { std::free(s); }

}  // extern "C"

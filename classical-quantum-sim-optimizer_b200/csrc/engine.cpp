#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <functional>
#include <map>
#include <mutex>
#include <thread>

#include <unistd.h>

#include "cost.hpp"

namespace dq {

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(kMemoryError, std::string("Unable to allocate device memory for ") + what);
    }
    fail(kCudaError, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

// Host worker threads shared by every parallel_for, started on first use and
// never torn down (they idle on a condition variable until the process ends).
// A call posts its job, works on it itself, then withdraws it and waits for
// the workers still inside one of its items; a worker only ever waits for
// items already running, so nested calls (an item that calls parallel_for)
// cannot deadlock.  A forked child, which has none of the workers, runs its
// calls on the calling thread.
class WorkerPool {
  public:
    struct Job {
        const std::function<void(size_t)>* fn = nullptr;
        size_t count = 0;
        std::atomic<size_t> next{0};
        int refs = 0;  // workers inside this job (guarded by the pool mutex)
        std::mutex error_mutex;
        std::exception_ptr error;
    };

    explicit WorkerPool(size_t workers) : owner_(getpid()) {
        for (size_t w = 0; w < workers; w++) std::thread([this] { loop(); }).detach();
    }

    // False in a process forked after the workers started.
    bool usable() const { return getpid() == owner_; }

    void run(Job& job) {
        {
            std::lock_guard<std::mutex> l(mutex_);
            jobs_.push_back(&job);
        }
        wake_.notify_all();
        work(job);
        std::unique_lock<std::mutex> l(mutex_);
        auto it = std::find(jobs_.begin(), jobs_.end(), &job);
        if (it != jobs_.end()) jobs_.erase(it);
        idle_.wait(l, [&] { return job.refs == 0; });
    }

  private:
    static void work(Job& job) {
        for (size_t i = job.next++; i < job.count; i = job.next++) {
            try {
                (*job.fn)(i);
            } catch (...) {
                std::lock_guard<std::mutex> l(job.error_mutex);
                if (!job.error) job.error = std::current_exception();
                job.next = job.count;
            }
        }
    }

    void loop() {
        std::unique_lock<std::mutex> l(mutex_);
        while (true) {
            wake_.wait(l, [&] { return !jobs_.empty(); });
            Job* job = jobs_.front();
            if (job->next.load() >= job->count) {
                jobs_.pop_front();
                continue;
            }
            job->refs++;
            l.unlock();
            work(*job);
            l.lock();
            if (--job->refs == 0) idle_.notify_all();
        }
    }

    const pid_t owner_;
    std::mutex mutex_;
    std::condition_variable wake_, idle_;
    std::deque<Job*> jobs_;
};

WorkerPool& worker_pool() {
    static WorkerPool* pool =
        new WorkerPool(std::min<size_t>(std::max<size_t>(1, std::thread::hardware_concurrency()), 16) - 1);
    return *pool;
}

}  // namespace

void parallel_for(size_t count, const std::function<void(size_t)>& fn) {
    if (count <= 1 || !worker_pool().usable()) {
        for (size_t i = 0; i < count; i++) fn(i);
        return;
    }
    WorkerPool::Job job;
    job.fn = &fn;
    job.count = count;
    worker_pool().run(job);
    if (job.error) std::rethrow_exception(job.error);
}

namespace {

// The engine's own stream-ordered memory pool per device: statevectors and
// sampling tables come from it, and freed blocks stay cached in it (release
// threshold: keep everything) so that repeated calls map no memory.  It is
// separate from the device's default pool, whose settings and cache belong to
// whatever else in the process uses cudaMallocAsync.
constexpr int kMaxPoolDevices = 64;
std::mutex g_devices_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};
// Live Device objects per ordinal: the pool is shared by every simulator (and
// result) on a device, so only the last one to go returns its cache.
std::map<int, int> g_devices_live;

cudaMemPool_t engine_pool(int dev) {
    std::lock_guard<std::mutex> l(g_devices_mu);
    if (dev < 0 || dev >= kMaxPoolDevices) fail(kValueError, "CUDA device ordinal out of range");
    if (!g_pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        cuda_check(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = ~uint64_t(0);
        cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep),
                   "memory pool release threshold");
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

// Returns the memory the current device's engine pool keeps cached.  Blocks
// freed on a stream return to the pool only once the stream reaches the free,
// so `sync_device` first waits for the whole device (the out-of-memory path,
// where another simulator's frees may still be pending).
void trim_pool(bool sync_device) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxPoolDevices) return;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> l(g_devices_mu);
        pool = g_pools[dev];
    }
    if (!pool) return;
    if (sync_device) cudaDeviceSynchronize();
    cudaMemPoolTrimTo(pool, 0);
}

}  // namespace

void DevMem::alloc(size_t b, const char* what) {
    release();
    if (b == 0) b = 16;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaErrorMemoryAllocation) {  // memory cached by the stream-ordered pool: give it back, retry
        cudaGetLastError();
        trim_pool(true);
        e = cudaMalloc(&p, b);
    }
    if (e != cudaSuccess) p = nullptr;
    cuda_check(e, what);
    bytes = b;
}

void DevMem::alloc_on(size_t b, cudaStream_t s, const char* what) {
    release();
    if (b == 0) b = 16;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cudaMemPool_t pool = engine_pool(dev);
    cudaError_t e = cudaMallocFromPoolAsync(&p, b, pool, s);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        trim_pool(true);
        e = cudaMallocFromPoolAsync(&p, b, pool, s);
    }
    if (e != cudaSuccess) p = nullptr;
    cuda_check(e, what);
    bytes = b;
    stream = s;
}

void DevMem::release() {
    if (p) {
        if (stream)
            cudaFreeAsync(p, stream);
        else
            cudaFree(p);
    }
    p = nullptr;
    bytes = 0;
    stream = nullptr;
}

Device::Device(int ord) : ordinal(ord) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        fail(kCudaError, std::string("no CUDA device available: ") + (e == cudaSuccess ? "0 devices" : cudaGetErrorString(e)));
    if (ord < 0 || ord >= count) fail(kValueError, "CUDA device ordinal out of range");
    cuda_check(cudaSetDevice(ord), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    engine_pool(ord);
    std::lock_guard<std::mutex> l(g_devices_mu);
    g_devices_live[ord]++;
}

Device::~Device() {
    if (stream) {
        cudaSetDevice(ordinal);
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
        bool last = false;
        {
            std::lock_guard<std::mutex> l(g_devices_mu);
            last = --g_devices_live[ordinal] == 0;
        }
        // Every other Device on this ordinal has synchronised and destroyed its
        // stream already, so the pool's pending frees have all completed.
        if (last) trim_pool(false);
    }
}

void Device::activate() const { cuda_check(cudaSetDevice(ordinal), "cudaSetDevice"); }

void Device::sync() { cuda_check(cudaStreamSynchronize(stream), "stream synchronize"); }

void StateBatch::allocate(int n_, uint64_t W_, uint64_t ncb_, bool c64_, cudaStream_t pool_stream) {
    n = n_;
    W = W_;
    ncb = ncb_;
    c64 = c64_;
    cwords = int(std::max<uint64_t>(1, (ncb + 63) / 64));
    // With a stream, every buffer comes from the engine's pool: freeing them
    // is stream-ordered and never waits for the device.
    auto get = [&](DevMem& m, size_t bytes, const char* what) {
        if (pool_stream)
            m.alloc_on(bytes, pool_stream, what);
        else
            m.alloc(bytes, what);
    };
    get(amps, (size_t(W) << n) * (c64 ? 8 : 16), "the statevector");
    get(cbits, size_t(W) * cwords * 8, "classical bits");
    get(seeds, size_t(W) * 8, "rng seeds");
    get(draws, size_t(W) * 8, "rng counters");
    get(outcome, size_t(W) * 4, "measurement outcomes");
    get(scale, size_t(W) * 8, "measurement scales");
    get(partial, size_t(W) * k::kMaxChunks * 2 * 8, "measurement partial sums");
    get(err, 16, "error flag");
}

k::Batch StateBatch::view(cudaStream_t s, uint64_t W_active) const {
    k::Batch b;
    b.stream = s;
    b.c64 = c64;
    b.amps = amps.p;
    b.n = n;
    b.W = W_active;
    b.cbits = cbits.as<uint64_t>();
    b.cwords = cwords;
    b.rng_seed = seeds.as<uint64_t>();
    b.draws = draws.as<uint64_t>();
    b.outcome = outcome.as<int>();
    b.scale = scale.as<double>();
    b.partial = partial.as<double>();
    b.err = err.as<int>();
    return b;
}

namespace {
double2 d2(cplx c) { return make_double2(c.re, c.im); }
}  // namespace

const char* kernel_class_name(int c) {
    static const char* names[kcNumClasses] = {"gate1q", "controlled", "diagonal", "swap", "dense",
                                              "measure", "tile", "fused", "sample", "norm"};
    return (c >= 0 && c < kcNumClasses) ? names[c] : "?";
}

EventRecorder::~EventRecorder() {
    for (auto& r : recs_) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : pool_) cudaEventDestroy(e);
}

cudaEvent_t EventRecorder::take() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    return e;
}

void EventRecorder::begin(int cls, double bytes, int kernels) {
    Rec r{cls, bytes, take(), take(), kernels};
    cuda_check(cudaEventRecord(r.a, stream_), "cudaEventRecord");
    recs_.push_back(r);
}

void EventRecorder::end() { cuda_check(cudaEventRecord(recs_.back().b, stream_), "cudaEventRecord"); }

void EventRecorder::collect(double* ms, uint64_t* launches, double* bytes) {
    cuda_check(cudaStreamSynchronize(stream_), "stream synchronize");
    for (int c = 0; c < kcNumClasses; c++) {
        ms[c] = 0;
        launches[c] = 0;
        bytes[c] = 0;
    }
    for (auto& r : recs_) {
        float t = 0;
        cuda_check(cudaEventElapsedTime(&t, r.a, r.b), "cudaEventElapsedTime");
        ms[r.cls] += t;
        launches[r.cls] += uint64_t(r.kernels);
        bytes[r.cls] += r.bytes;
        pool_.push_back(r.a);
        pool_.push_back(r.b);
    }
    recs_.clear();
}

double Executor::step_bytes(size_t i, const k::Batch& b) const {
    const Step& s = steps_[i];
    const double S = b.c64 ? 8.0 : 16.0;
    const double full = S * double(uint64_t(1) << b.n) * double(b.W);
    if (s.pass >= 0 || s.fused >= 0) return 2.0 * full;
    switch (s.type) {
        case Operation::One:
        case Operation::X: return 2.0 * full / double(uint64_t(1) << s.controls.size());
        case Operation::Swap: return full / double(uint64_t(1) << s.controls.size());
        case Operation::Diagonal: {
            int kq = int(s.qubits.size()), e = 0;
            for (auto& d : s.diag)
                if (!(d.x == 1.0 && d.y == 0.0)) e++;
            if (e * 2 <= (1 << kq)) return 2.0 * full * e / double(1 << kq);
            return 2.0 * full;
        }
        case Operation::Dense: return 2.0 * full;
        case Operation::Measure:
        case Operation::Reset: return 2.5 * full;
        default: return 0.0;
    }
}

namespace {
// Real operations of a 2^k x 2^k complex matrix-vector product.
double dense_flops(int k) {
    const double d = double(1 << k);
    return d * d * 6.0 + (d * d - d) * 2.0;
}
}  // namespace

void Executor::arith_flops(const k::Batch& b, double* cuda_core, double* tensor) const {
    const double amps = double(uint64_t(1) << b.n) * double(b.W);
    double cc = 0.0, tc = 0.0;
    for (const Step& s : steps_) {
        if (s.fused >= 0) {
            const FusedPass& p = fused_[size_t(s.fused)];
            tc += double(p.nblocks) * (amps / double(1 << kFusedM)) * 3.0 * 2.0 * 128.0 * 64.0 * 64.0;
            continue;
        }
        if (s.pass >= 0) {
            const TilePass& p = passes_[size_t(s.pass)];
            const int m = int(p.qubits.size());
            const double tiles = amps / double(uint64_t(1) << m);
            double per_tile = 0.0;
            for (const TileOp& op : p.ops) {
                const double items = double(uint64_t(1) << (m - op.nins));
                switch (op.type) {
                    case TileOp::kOne: per_tile += items * 28.0; break;
                    case TileOp::kDiagEntry: per_tile += items * 6.0; break;
                    case TileOp::kDiagFull: per_tile += double(uint64_t(1) << m) * 6.0; break;
                    case TileOp::kDense: per_tile += double(uint64_t(1) << (m - op.k)) * dense_flops(op.k); break;
                    default: break;  // X and swap move amplitudes only
                }
            }
            cc += tiles * per_tile;
            continue;
        }
        const double pairs = amps / 2.0 / double(uint64_t(1) << s.controls.size());
        switch (s.type) {
            case Operation::One: cc += pairs * 28.0; break;
            case Operation::Diagonal: {
                const int kq = int(s.qubits.size());
                double e = 0;
                for (auto& d : s.diag)
                    if (!(d.x == 1.0 && d.y == 0.0)) e++;
                cc += amps / double(1 << kq) * e * 6.0;
                break;
            }
            case Operation::Dense: cc += amps / double(1 << s.qubits.size()) * dense_flops(int(s.qubits.size())); break;
            case Operation::Measure:
            case Operation::Reset: cc += amps * 5.0; break;  // |a|^2 sums, then one scale per kept amplitude
            default: break;
        }
    }
    *cuda_core = cc;
    *tensor = tc;
}

Executor::Executor(const std::vector<Operation>& ops, size_t begin, size_t end, const ExecConfig& cfg) : cfg_(cfg) {
    size_t seg = begin;
    if (cfg_.fuse > kTileMaxDense) cfg_.fuse = kTileMaxDense;
    for (size_t i = begin; i < end; i++) {
        if (cfg_.tiled && tileable(ops[i])) continue;
        if (seg < i) lower_segment(ops, seg, i);
        std::vector<Condition> conds;
        lower(ops[i], conds);
        seg = i + 1;
    }
    if (seg < end) lower_segment(ops, seg, end);
}

void Executor::lower_segment(const std::vector<Operation>& ops, size_t begin, size_t end) {
    if (!cfg_.tiled || cfg_.n < 1) {
        for (size_t i = begin; i < end; i++) {
            std::vector<Condition> conds;
            lower(ops[i], conds);
        }
        return;
    }
    TilePlanOptions o;
    o.m = cfg_.tile_m;
    o.fuse = cfg_.fuse;
    o.seeds = cfg_.seeds;
    o.beam = kPlanBeam;
    o.c64 = cfg_.c64;
    o.model = cfg_.model;
    o.chosen_widths = &widths_;
    if (cfg_.fused && cfg_.c64 && cfg_.n >= kFusedM) {
        std::vector<BuiltFusedPass> built;
        {
            FusedPlanChoice ch;
            FusedPortfolio pf = fused_portfolio(ops, begin, end, cfg_.n, o, fused_caps(cfg_.n, cfg_.pass_model != nullptr));
            ch.caps = pf.caps;
            ch.rule_cost = pf.rule_cost;
            ch.rule_choice = ch.chosen = pf.rule_choice;
            for (size_t i = 0; i < pf.plans.size(); i++) {
                size_t nb = 0;
                for (size_t slot : pf.slots[i]) nb += size_t(pf.built[slot].fp.nblocks);
                ch.passes.push_back(pf.plans[i].size());
                ch.blocks.push_back(nb);
            }
            if (cfg_.pass_model) {
                // The learned pass-cost model picks the plan of least predicted time.
                ch.predicted_ms = cfg_.pass_model->predict_plans_ms(pf, 1);
                for (size_t i = 0; i < ch.predicted_ms.size(); i++)
                    if (ch.predicted_ms[i] < ch.predicted_ms[ch.chosen]) ch.chosen = i;
            }
            built = take_fused_plan(pf, ch.chosen);
            fused_choices_.push_back(std::move(ch));
        }
        // With a trained cost model each pass runs on whichever executor it
        // predicts cheapest: tensor-core blocks (0) or CUDA-core tile operations
        // fused to width 1..kTileMaxDense.
        std::vector<int> choices(built.size(), 0);
        if (cfg_.model)
            parallel_for(built.size(), [&](size_t i) {
                const BuiltFusedPass& bt = built[i];
                double best = cfg_.model->predict_fused(bt.fp);
                for (int w = 1; w <= kTileMaxDense; w++) {
                    std::vector<double2> scratch;
                    std::vector<TileOp> cand;
                    lower_pass_ops(bt.src.raw, bt.src.qubits, cfg_.n, w, scratch, cand);
                    const double cost = cfg_.model->predict_ops(cand, kFusedM, true);
                    if (cost < best) {
                        best = cost;
                        choices[i] = w;
                    }
                }
            });
        for (size_t i = 0; i < built.size(); i++) {
            BuiltFusedPass& bt = built[i];
            TilePass& p = bt.src;
            const int choice = choices[i];
            widths_.push_back(choice);
            Step s;
            s.type = Operation::Dense;
            s.category = 1;
            if (choice == 0) {
                s.fused = int(fused_.size());
                bt.fp.first_block += int(fused_blocks_host_.size());
                for (FusedBlock& fb : bt.blocks) fb.u_off += uint32_t(upool_host_.size());
                fused_blocks_host_.insert(fused_blocks_host_.end(), bt.blocks.begin(), bt.blocks.end());
                upool_host_.insert(upool_host_.end(), bt.upool.begin(), bt.upool.end());
                fused_.push_back(std::move(bt.fp));
                fused_src_.push_back(std::move(p));
            } else {
                lower_pass_ops(p.raw, p.qubits, cfg_.n, choice, pool_host_, p.ops);
                p.raw.clear();
                p.op_begin = int(tile_ops_host_.size());
                tile_ops_host_.insert(tile_ops_host_.end(), p.ops.begin(), p.ops.end());
                attach_phases(p);
                s.pass = int(passes_.size());
                passes_.push_back(std::move(p));
            }
            steps_.push_back(std::move(s));
        }
        return;
    }
    std::vector<TilePass> ps = plan_tiles(ops, begin, end, cfg_.n, o, &pool_host_);
    for (auto& p : ps) {
        p.op_begin = int(tile_ops_host_.size());
        tile_ops_host_.insert(tile_ops_host_.end(), p.ops.begin(), p.ops.end());
        attach_phases(p);
        Step s;
        s.pass = int(passes_.size());
        s.type = Operation::Dense;
        s.category = 1;
        passes_.push_back(std::move(p));
        steps_.push_back(std::move(s));
    }
}

void Executor::attach_phases(TilePass& p) {
    const int m = int(p.qubits.size());
    // complex128 only: on complex64 tiles the phases measured slower than one
    // operation per sweep (FP32 arithmetic leaves shared memory less of the time).
    if (!cfg_.phased || cfg_.c64 || cfg_.model || !phase_supported(m) || p.ops.empty()) return;
    std::vector<uint4> block;
    p.nphases = plan_phases(p.ops, m, cfg_.c64, pool_host_, block);
    p.phase_block = int(phase_blocks_.size());
    p.phase_begin = int(phase_words_host_.size());
    phase_words_host_.insert(phase_words_host_.end(), block.begin(), block.end());
    phase_blocks_.push_back(std::move(block));
}

void Executor::record_costs(const k::Batch& b, std::vector<float>& X, std::vector<float>& y) {
    run(b, nullptr, nullptr);  // uploads the pools; the state it leaves is reused below
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    // Device milliseconds of one launch sequence (the faster of two runs).
    auto time_ms = [&](auto&& launch) {
        float best = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            cuda_check(cudaEventRecord(e0, b.stream), "cudaEventRecord");
            launch();
            cuda_check(cudaEventRecord(e1, b.stream), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            best = std::min(best, ms);
        }
        return double(best);
    };
    DevMem cyc, tops, tpool;
    std::vector<unsigned long long> host;
    // One CUDA-core pass: its event time shared among its operations by cycles.
    auto record_tile = [&](const TilePass& p, const TileOp* ops_dev, const double2* pool_dev,
                           const std::vector<TileOp>& ops_host) {
        if (ops_host.empty()) return;
        const int m = int(p.qubits.size());
        const int nops = int(ops_host.size());
        const double tiles = double(b.W << (b.n - m));
        const double ms = time_ms([&] { k::tile_pass(b, nullptr, m, ops_dev, nops, pool_dev, p, nullptr); });
        cyc.ensure(size_t(nops) * 8, "cycle counters");
        cuda_check(cudaMemsetAsync(cyc.p, 0, size_t(nops) * 8, b.stream), "clear cycle counters");
        k::tile_pass(b, nullptr, m, ops_dev, nops, pool_dev, p, cyc.as<unsigned long long>());
        host.resize(size_t(nops));
        cuda_check(cudaMemcpyAsync(host.data(), cyc.p, size_t(nops) * 8, cudaMemcpyDeviceToHost, b.stream), "read");
        cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
        double total = 0;
        for (auto c : host) total += double(std::max<unsigned long long>(c, 1));
        for (int i = 0; i < nops; i++) {
            float f[kMlpF];
            tile_op_features(ops_host[size_t(i)], m, b.c64, f);
            X.insert(X.end(), f, f + kMlpF);
            const double share = double(std::max<unsigned long long>(host[size_t(i)], 1)) / total;
            y.push_back(float(std::log(std::max(1.0, ms * 1e9 / tiles * share))));
        }
    };
    for (size_t si = 0; si < steps_.size(); si++) {
        const Step& s = steps_[si];
        if (s.pass >= 0) {
            const TilePass& p = passes_[size_t(s.pass)];
            record_tile(p, tile_ops_.as<TileOp>() + p.op_begin, pool_.as<double2>(), p.ops);
        } else if (s.fused >= 0) {
            const FusedPass& fp = fused_[size_t(s.fused)];
            const double tiles = double(b.W << (b.n - kFusedM));
            norm_tiles_.ensure(size_t(tiles) * 8, "fused tile norms");
            const double ms = time_ms([&] {
                k::fused_pass(b, fp, fused_blocks_.as<FusedBlock>(), upool_.as<uint16_t>(), b.err, nullptr,
                              norm_tiles_.as<double>());
            });
            for (int j = 0; j < fp.nblocks; j++) {
                float f[kMlpF];
                fused_block_features(fp.block_gates[size_t(j)], fp.block_masks[size_t(j)], fp.nblocks, f);
                X.insert(X.end(), f, f + kMlpF);
                y.push_back(float(std::log(std::max(1.0, ms * 1e9 / tiles / fp.nblocks))));
            }
            // The same pass on CUDA cores at each fusion width.
            const TilePass& src = fused_src_[size_t(s.fused)];
            for (int w = 1; w <= kTileMaxDense; w++) {
                std::vector<double2> pool;
                std::vector<TileOp> ops;
                lower_pass_ops(src.raw, src.qubits, b.n, w, pool, ops);
                if (ops.empty()) continue;
                tops.ensure(ops.size() * sizeof(TileOp), "tile operations");
                tpool.ensure(std::max<size_t>(pool.size(), 1) * sizeof(double2), "gate matrices");
                cuda_check(cudaMemcpyAsync(tops.p, ops.data(), ops.size() * sizeof(TileOp), cudaMemcpyHostToDevice,
                                           b.stream),
                           "upload tile operations");
                if (!pool.empty())
                    cuda_check(cudaMemcpyAsync(tpool.p, pool.data(), pool.size() * sizeof(double2),
                                               cudaMemcpyHostToDevice, b.stream),
                               "upload gate matrices");
                record_tile(src, tops.as<TileOp>(), tpool.as<double2>(), ops);
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // The timed passes left the state arbitrary and its norm unchecked.
    cuda_check(cudaMemsetAsync(b.err, 0, 16, b.stream), "clear error flag");
    cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
}

size_t Executor::raw_ops_in_passes() const {
    size_t t = 0;
    for (auto& p : passes_) t += size_t(p.raw_ops);
    return t;
}

void Executor::lower(const Operation& op, std::vector<Condition>& conds) {
    if (op.type == Operation::Conditional) {
        conds.push_back(op.condition);
        lower(*op.inner, conds);
        conds.pop_back();
        return;
    }
    if (op.type == Operation::Noop) return;
    if (conds.size() > 6) fail(kValueError, "Classical conditions nested deeper than 6 levels are not supported");
    Step s;
    s.type = op.type;
    s.host_conds = conds;
    s.cond.n = int(conds.size());
    for (size_t i = 0; i < conds.size(); i++) {
        s.cond.base[i] = conds[i].creg_base;
        s.cond.size[i] = uint32_t(conds[i].creg_size);
        s.cond.value[i] = conds[i].creg_value;
    }
    for (auto& c : op.controls) s.controls.push_back({int(c.qubit), c.value});
    switch (op.type) {
        case Operation::One:
            s.target = int(op.target);
            s.u[0] = d2(op.m[0][0]);
            s.u[1] = d2(op.m[0][1]);
            s.u[2] = d2(op.m[1][0]);
            s.u[3] = d2(op.m[1][1]);
            s.category = op.controls.empty() ? 0 : 1;
            break;
        case Operation::X:
            s.target = int(op.target);
            s.category = op.controls.empty() ? 0 : 1;
            break;
        case Operation::Swap:
            s.a = int(op.a);
            s.b = int(op.b);
            s.category = 1;
            break;
        case Operation::Diagonal:
            for (auto q : op.qubits) s.qubits.push_back(int(q));
            for (auto& v : op.values) s.diag.push_back(d2(v));
            s.category = op.qubits.size() > 1 ? 1 : 0;
            break;
        case Operation::Dense:
            for (auto q : op.qubits) s.qubits.push_back(int(q));
            s.pool_offset = pool_host_.size();
            for (auto& v : op.values) pool_host_.push_back(d2(v));
            s.category = 1;
            break;
        case Operation::Measure:
            s.target = int(op.qubit);
            s.cbit = int64_t(op.cbit);
            s.category = 2;
            break;
        case Operation::Reset:
            s.target = int(op.qubit);
            s.cbit = -1;
            s.category = 2;
            break;
        default: fail(kValueError, "unexpected operation");
    }
    steps_.push_back(std::move(s));
}

void Executor::prepare(const k::Batch& b) {
    if (!fused_.empty()) {
        norm_tiles_.ensure((size_t(b.W) << (b.n - kFusedM)) * 8, "fused tile norms");
        norm_states_.ensure(size_t(b.W) * size_t(k::fused_norm_parts(b.n)) * 8, "fused state norms");
        k::fused_configure();
    }
    upload(b.stream);
}

void Executor::upload(cudaStream_t stream) {
    if (uploaded_) return;
    if (!pool_host_.empty()) {
        pool_.alloc(pool_host_.size() * sizeof(double2), "gate matrices");
        cuda_check(cudaMemcpyAsync(pool_.p, pool_host_.data(), pool_host_.size() * sizeof(double2),
                                   cudaMemcpyHostToDevice, stream),
                   "upload gate matrices");
    }
    if (!tile_ops_host_.empty()) {
        tile_ops_.alloc(tile_ops_host_.size() * sizeof(TileOp), "tile operations");
        cuda_check(cudaMemcpyAsync(tile_ops_.p, tile_ops_host_.data(), tile_ops_host_.size() * sizeof(TileOp),
                                   cudaMemcpyHostToDevice, stream),
                   "upload tile operations");
    }
    if (!phase_words_host_.empty()) {
        phase_words_.alloc(phase_words_host_.size() * sizeof(uint4), "tile phases");
        cuda_check(cudaMemcpyAsync(phase_words_.p, phase_words_host_.data(), phase_words_host_.size() * sizeof(uint4),
                                   cudaMemcpyHostToDevice, stream),
                   "upload tile phases");
    }
    if (!fused_blocks_host_.empty()) {
        fused_blocks_.alloc(fused_blocks_host_.size() * sizeof(FusedBlock), "fused block descriptors");
        upool_.alloc(upool_host_.size() * sizeof(uint16_t), "fused block gate images");
        cuda_check(cudaMemcpyAsync(fused_blocks_.p, fused_blocks_host_.data(),
                                   fused_blocks_host_.size() * sizeof(FusedBlock), cudaMemcpyHostToDevice, stream),
                   "upload fused blocks");
        cuda_check(cudaMemcpyAsync(upool_.p, upool_host_.data(), upool_host_.size() * sizeof(uint16_t),
                                   cudaMemcpyHostToDevice, stream),
                   "upload gate images");
    }
    uploaded_ = true;
}

void Executor::run(const k::Batch& b, ProfileAcc* profile, EventRecorder* rec, bool normalize, bool from_basis) {
    upload(b.stream);
    std::vector<uint64_t> host_cbits;
    bool norm_pending = false;  // a fused pass left a norm the next fused pass divides out
    for (size_t si = 0; si < steps_.size(); si++) {
        const Step& s = steps_[si];
        if (profile && s.cond.n) {
            // Profiling counts only executed operations (execution.rs:285-295),
            // so the host reads the single trajectory's classical bits here.
            host_cbits.resize(size_t(b.cwords));
            cuda_check(cudaMemcpyAsync(host_cbits.data(), b.cbits, size_t(b.cwords) * 8, cudaMemcpyDeviceToHost,
                                       b.stream),
                       "read classical bits");
            cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
            bool ok = true;
            for (auto& c : s.host_conds) {
                uint64_t v = 0;
                for (uint64_t bit = 0; bit < c.creg_size; bit++) {
                    uint64_t idx = c.creg_base + bit;
                    v |= ((host_cbits[idx >> 6] >> (idx & 63)) & 1) << bit;
                }
                if (v != c.creg_value) ok = false;
            }
            if (!ok) continue;
        }
        auto t0 = std::chrono::steady_clock::now();
        if (s.fused >= 0) {
            const FusedPass& p = fused_[size_t(s.fused)];
            const size_t tiles = size_t(b.W) << (b.n - kFusedM);
            norm_tiles_.ensure(tiles * 8, "fused tile norms");
            norm_states_.ensure(size_t(b.W) * size_t(k::fused_norm_parts(b.n)) * 8, "fused state norms");
            if (rec) rec->begin(kcFused, step_bytes(si, b));
            k::fused_pass(b, p, fused_blocks_.as<FusedBlock>(), upool_.as<uint16_t>(), b.err,
                          norm_pending ? norm_states_.as<double>() : nullptr, norm_tiles_.as<double>(),
                          from_basis && si == 0);
            if (rec) rec->end();
            const bool last_fused = si + 1 == steps_.size() || steps_[si + 1].fused < 0;
            if (normalize || si + 1 != steps_.size()) {
                // Tile norms read (8 B per tile); the final rescale reads and writes the state.
                if (rec)
                    rec->begin(kcNorm,
                               double(tiles) * 8.0 + (last_fused ? 2.0 * double(size_t(b.W) << b.n) * 8.0 : 0.0),
                               last_fused ? 2 : 1);
                k::fused_state_norm(b, norm_tiles_.as<double>(), norm_states_.as<double>());
                norm_pending = true;
                if (last_fused) {
                    k::fused_renormalize(b, norm_states_.as<double>());
                    norm_pending = false;
                }
                if (rec) rec->end();
            }
            if (profile) {
                cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
                profile->nq_calls++;
                profile->nq_time += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            }
            continue;
        }
        if (s.pass >= 0) {
            const TilePass& p = passes_[size_t(s.pass)];
            if (rec) rec->begin(kcTile, step_bytes(si, b));
            const int m = int(p.qubits.size());
            if (p.nphases > 0)
                k::tile_pass_phased(b, p, p.nphases, phase_blocks_[size_t(p.phase_block)],
                                    phase_words_.as<uint4>() + p.phase_begin);
            else
                k::tile_pass(b, nullptr, m, tile_ops_.as<TileOp>() + p.op_begin, int(p.ops.size()),
                             pool_.as<double2>(), p);
            if (rec) rec->end();
            if (profile) {
                cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
                profile->nq_calls++;
                profile->nq_time += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            }
            continue;
        }
        if (rec) {
            int cls = kcGate1q;
            switch (s.type) {
                case Operation::One: cls = s.controls.empty() ? kcGate1q : kcControlled; break;
                case Operation::X: cls = kcControlled; break;
                case Operation::Swap: cls = kcSwap; break;
                case Operation::Diagonal: cls = kcDiagonal; break;
                case Operation::Dense: cls = kcDense; break;
                default: cls = kcMeasure; break;
            }
            rec->begin(cls, step_bytes(si, b));
        }
        switch (s.type) {
            case Operation::One: k::gate1q(b, s.target, s.controls, s.u, false, s.cond); break;
            case Operation::X: k::gate1q(b, s.target, s.controls, s.u, true, s.cond); break;
            case Operation::Swap: k::swap(b, s.a, s.b, s.controls, s.cond); break;
            case Operation::Diagonal: k::diagonal(b, s.qubits, s.diag, s.cond); break;
            case Operation::Dense: k::dense(b, s.qubits, pool_.as<double2>() + s.pool_offset, s.cond); break;
            case Operation::Measure: k::measure(b, s.target, s.cbit, false, s.cond); break;
            case Operation::Reset: k::measure(b, s.target, -1, true, s.cond); break;
            default: break;
        }
        if (rec) rec->end();
        if (profile) {
            cuda_check(cudaStreamSynchronize(b.stream), "stream synchronize");
            double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (s.category == 0) {
                profile->oq_calls++;
                profile->oq_time += dt;
            } else if (s.category == 1) {
                profile->nq_calls++;
                profile->nq_time += dt;
            } else {
                profile->mq_calls++;
                profile->mq_time += dt;
            }
        }
    }
}

}  // namespace dq

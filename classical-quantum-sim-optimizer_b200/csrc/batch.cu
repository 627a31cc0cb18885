#include "batch.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "device.cuh"

namespace dq {
namespace {

constexpr int kBatchThreads = 256;
// Side streams the fused circuits of a batch run on.
constexpr size_t kSideStreams = 16;
// Spin limit of one dependency wait: 2^24 polls of >= 256 ns, several seconds.
constexpr uint64_t kMaxSpins = uint64_t(1) << 24;

template <typename V>
__device__ __forceinline__ V ld_cg(const V* p);
template <>
__device__ __forceinline__ double2 ld_cg<double2>(const double2* p) {
    return __ldcg(p);
}
template <>
__device__ __forceinline__ float2 ld_cg<float2>(const float2* p) {
    return __ldcg(p);
}

// The per-operation semantics are those of the single-circuit tile pass.
__device__ __forceinline__ uint32_t expand_local(uint32_t j, const TileOp& op) {
#pragma unroll
    for (int t = 0; t < 7; t++) {
        if (t < op.nins) {
            uint32_t low = (1u << op.ins[t]) - 1;
            j = (j & low) | ((j & ~low) << 1);
        }
    }
    return j;
}

template <typename V, int K>
__device__ void b_dense(V* __restrict__ tile, const TileOp& op, int m, const double2* __restrict__ pool) {
    constexpr int D = 1 << K;
    const uint32_t items = 1u << (m - K);
    const double2* mat = pool + op.mat;
    for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
        const uint32_t base = expand_local(j, op);
        V v[D];
#pragma unroll
        for (int c = 0; c < D; c++) v[c] = tile[base | op.offs[c]];
#pragma unroll 1
        for (int r = 0; r < D; r++) {
            V acc = dev::czero<V>();
#pragma unroll
            for (int c = 0; c < D; c++) acc = dev::cadd(acc, dev::cmul(dev::from_d2<V>(__ldg(mat + r * D + c)), v[c]));
            tile[base | op.offs[r]] = acc;
        }
    }
}

template <typename V>
__device__ void b_apply(V* __restrict__ tile, const TileOp& op, int m, const double2* __restrict__ pool) {
    switch (op.type) {
        case TileOp::kOne:
        case TileOp::kX: {
            const uint32_t items = 1u << (m - op.nins);
            const bool is_x = op.type == TileOp::kX;
            V u00 = dev::czero<V>(), u01 = u00, u10 = u00, u11 = u00;
            if (!is_x) {
                u00 = dev::from_d2<V>(__ldg(pool + op.mat));
                u01 = dev::from_d2<V>(__ldg(pool + op.mat + 1));
                u10 = dev::from_d2<V>(__ldg(pool + op.mat + 2));
                u11 = dev::from_d2<V>(__ldg(pool + op.mat + 3));
            }
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i0 = expand_local(j, op) | op.fixed, i1 = i0 | op.tbit;
                V a = tile[i0], b = tile[i1];
                if (is_x) {
                    tile[i0] = b;
                    tile[i1] = a;
                } else {
                    tile[i0] = dev::cadd(dev::cmul(u00, a), dev::cmul(u01, b));
                    tile[i1] = dev::cadd(dev::cmul(u10, a), dev::cmul(u11, b));
                }
            }
            break;
        }
        case TileOp::kDiagEntry: {
            const uint32_t items = 1u << (m - op.nins);
            const V v = dev::from_d2<V>(__ldg(pool + op.mat));
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i = expand_local(j, op) | op.fixed;
                tile[i] = dev::cmul(tile[i], v);
            }
            break;
        }
        case TileOp::kDiagFull: {
            const uint32_t items = 1u << m;
            for (uint32_t i = threadIdx.x; i < items; i += blockDim.x) {
                uint32_t jj = 0;
                for (int b = 0; b < op.k; b++) jj = (jj << 1) | ((i >> op.q[b]) & 1u);
                tile[i] = dev::cmul(tile[i], dev::from_d2<V>(__ldg(pool + op.mat + jj)));
            }
            break;
        }
        case TileOp::kSwap: {
            const uint32_t items = 1u << (m - op.nins);
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i = expand_local(j, op) | op.fixed;
                V a = tile[i | op.lowbit];
                tile[i | op.lowbit] = tile[i | op.highbit];
                tile[i | op.highbit] = a;
            }
            break;
        }
        case TileOp::kDense:
            switch (op.k) {
                case 1: b_dense<V, 1>(tile, op, m, pool); break;
                case 2: b_dense<V, 2>(tile, op, m, pool); break;
                case 3: b_dense<V, 3>(tile, op, m, pool); break;
            }
            break;
    }
}

template <typename V>
__global__ void __launch_bounds__(kBatchThreads) k_batch(V* __restrict__ amps, const BatchRun::PassRec* __restrict__ recs,
                                                         int nrecs, const TileOp* __restrict__ ops,
                                                         const double2* __restrict__ pool,
                                                         unsigned long long* __restrict__ done,
                                                         unsigned long long* __restrict__ head, uint64_t total,
                                                         int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t s_item;
    __shared__ int s_rec, s_abort;
    __shared__ uint64_t lo_tab[64];
    __shared__ uint64_t hi_tab[1 << 8];  // tiles hold at most 14 qubits
    V* tile = reinterpret_cast<V*>(smem_raw);
    while (true) {
        if (threadIdx.x == 0) {
            s_abort = 0;
            s_item = atomicAdd(head, 1ULL);
            if (s_item < total) {
                int lo = 0, hi = nrecs - 1;  // last record with item_begin <= item
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (recs[mid].item_begin <= s_item)
                        lo = mid;
                    else
                        hi = mid - 1;
                }
                s_rec = lo;
                const BatchRun::PassRec& R = recs[lo];
                // Wait until every tile of the circuit's earlier passes is written back.
                volatile unsigned long long* cnt = done + R.circuit;
                uint64_t spins = 0;
                while (*cnt < R.wait_count) {
                    if (++spins > kMaxSpins || *(volatile int*)err) {
                        atomicExch(err, 2);
                        s_abort = 1;
                        break;
                    }
                    __nanosleep(256);
                }
                __threadfence();
            }
        }
        __syncthreads();
        const uint64_t item = s_item;
        if (item >= total || s_abort) break;
        const BatchRun::PassRec& R = recs[s_rec];
        const int m = R.m, n = R.n;
        const int lb = m < 6 ? m : 6;
        for (int e = threadIdx.x; e < (1 << lb); e += blockDim.x) {
            uint64_t off = 0;
            for (int b = 0; b < lb; b++)
                if ((e >> b) & 1) off |= uint64_t(1) << R.q[b];
            lo_tab[e] = off;
        }
        for (int e = threadIdx.x; e < (1 << (m - lb)); e += blockDim.x) {
            uint64_t off = 0;
            for (int b = 0; b < m - lb; b++)
                if ((e >> b) & 1) off |= uint64_t(1) << R.q[lb + b];
            hi_tab[e] = off;
        }
        uint64_t tid = item - R.item_begin;
        for (int b = 0; b < m; b++) {
            uint64_t low = (uint64_t(1) << R.q[b]) - 1;
            tid = (tid & low) | ((tid & ~low) << 1);
        }
        (void)n;
        V* __restrict__ g = amps + R.state_off + tid;
        __syncthreads();
        const uint32_t size = 1u << m, lmask = (1u << lb) - 1;
        for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) tile[e] = ld_cg<V>(g + (lo_tab[e & lmask] | hi_tab[e >> lb]));
        __syncthreads();
        for (int i = 0; i < R.nops; i++) {
            b_apply<V>(tile, ops[R.op_begin + i], m, pool);
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) __stcg(g + (lo_tab[e & lmask] | hi_tab[e >> lb]), tile[e]);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done + R.circuit, 1ULL);
        }
    }
}

template <typename V>
__global__ void k_first_amp(V* amps, const uint64_t* __restrict__ offs, int count) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < count) {
        V one = dev::czero<V>();
        one.x = 1;
        amps[offs[c]] = one;
    }
}

template <typename V>
__global__ void k_arena_norm2(const V* __restrict__ amps, double* __restrict__ out, uint64_t len) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x)
        out[g] = dev::norm2(amps[g]);
}

// <Z0 Z1> per circuit from its probabilities (one block per circuit, fixed-order tree).
__global__ void k_zz(const double* __restrict__ probs, const uint64_t* __restrict__ offs, int count,
                     double* __restrict__ out) {
    __shared__ double sm[256];
    const int c = blockIdx.x;
    const uint64_t b = offs[c], e = offs[count + c];
    double acc = 0.0;
    for (uint64_t i = threadIdx.x; i < e - b; i += blockDim.x) {
        double p = probs[b + i];
        acc += ((i ^ (i >> 1)) & 1) ? -p : p;
    }
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sm[0];
}

// base/total of each circuit's segment of the global inclusive scan.
__global__ void k_seg_totals(const double* __restrict__ scan, const uint64_t* __restrict__ offs, int count,
                             double* __restrict__ base_total, int* __restrict__ err) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    uint64_t b = offs[c], e = offs[count + c];
    double base = b > 0 ? scan[b - 1] : 0.0;
    double tot = scan[e - 1] - base;
    if (!(isfinite(tot) && tot > 0.0)) atomicExch(err, 1);
    base_total[2 * c] = base;
    base_total[2 * c + 1] = tot;
}

__global__ void k_seg_normalize(double* __restrict__ cdf, const uint64_t* __restrict__ offs, int count,
                                const double* __restrict__ base_total) {
    int c = blockIdx.y;
    uint64_t b = offs[c], e = offs[count + c];
    double base = base_total[2 * c], tot = base_total[2 * c + 1];
    for (uint64_t i = b + uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < e; i += uint64_t(gridDim.x) * blockDim.x)
        cdf[i] = (i == e - 1) ? 1.0 : (cdf[i] - base) / tot;
}

__global__ void k_seg_sample(const double* __restrict__ cdf, const uint64_t* __restrict__ offs, int count,
                             const uint64_t* __restrict__ seeds, uint64_t shots, uint64_t* __restrict__ out) {
    uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= uint64_t(count) * shots) return;
    int c = int(g / shots);
    uint64_t t = g % shots;
    uint64_t b = offs[c], e = offs[count + c];
    double draw = dev::u64_to_unit(dev::chacha8_u64(seeds[c] + t, 0));
    uint64_t lo = b, hi = e;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] <= draw)
            lo = mid + 1;
        else
            hi = mid;
    }
    uint64_t idx = lo - b;
    out[g] = idx < e - b - 1 ? idx : e - b - 1;
}

int sm_count() {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c > 0 ? c : 148;
}

}  // namespace

BatchRun::BatchRun(Simulator& sim, const std::vector<std::string>& texts, uint64_t shots, const BatchTuning& tuning)
    : shots_(shots) {
    const Options& o = sim.options();
    c64_ = o.precision == Precision::C64;
    std::vector<std::vector<TilePass>> plans;
    uint64_t off = 0;
    for (size_t ci = 0; ci < texts.size(); ci++) {
        Circ c;
        std::vector<Operation> ops = compile_json(texts[ci].data(), texts[ci].size(), &c.n, &c.ncb);
        if (c.n > 30) fail(kValueError, "batched circuits are limited to 30 qubits each");
        size_t prefix = ops.size();
        for (size_t i = 0; i < ops.size(); i++)
            if (!ops[i].is_unitary()) {
                prefix = i;
                break;
            }
        std::map<uint64_t, uint64_t> mapping;
        for (size_t i = prefix; i < ops.size(); i++) {
            if (ops[i].type != Operation::Measure)
                fail(kValueError, "batched circuits must end in measurements only (mid-circuit measurement, reset "
                                  "and classical control run through simulate_shots)");
            mapping[ops[i].cbit] = ops[i].qubit;
        }
        for (size_t i = 0; i < prefix; i++)
            if (!tileable(ops[i])) fail(kValueError, "batched circuits support gates of at most 3 dense qubits");
        // Sampling runs over the full register; measured qubits are read from the sampled index.
        for (auto& kv : mapping) c.cbit_map.emplace_back(kv.first, kv.second);
        c.tile_m = tuning.tile_m > 0 ? tuning.tile_m : (c64_ ? 13 : 12);
        c.fuse = tuning.fuse > 0 ? tuning.fuse : 2;
        c.depth = tuning.depth;
        auto tuned = tuning.per_n.find(c.n);
        if (tuning.tile_m <= 0 && tuning.fuse <= 0 && tuned != tuning.per_n.end()) {
            c.tile_m = tuned->second.tile_m;
            c.fuse = tuned->second.fuse;
            c.depth = tuned->second.depth;
        }
        std::vector<TilePass> passes;
        if (c.fuse == 5 && c64_ && c.n >= uint64_t(kFusedM)) {
            // Tensor-core fused passes, run by an executor of their own on a side stream.
            ExecConfig cfg;
            cfg.tiled = true;
            cfg.fused = true;
            cfg.c64 = true;
            cfg.n = int(c.n);
            c.fused = std::make_unique<Executor>(ops, 0, prefix, cfg);
        } else {
            if (c.fuse == 5) c.fuse = 2;  // no tensor-core form below 12 qubits or in complex128
            TilePlanOptions po;
            po.m = c.tile_m;
            po.fuse = std::min(c.fuse, kTileMaxDense);
            po.c64 = c64_;
            po.max_pass_ops = c.depth;
            passes = plan_tiles(ops, 0, prefix, int(c.n), po, &pool_host_);
            for (auto& p : passes) {
                p.op_begin = int(ops_host_.size());
                ops_host_.insert(ops_host_.end(), p.ops.begin(), p.ops.end());
                max_m_ = std::max(max_m_, int(p.qubits.size()));
            }
        }
        c.state_off = off;
        off += uint64_t(1) << c.n;
        off = (off + 255) & ~uint64_t(255);
        c.seed = (o.has_seed ? o.seed : 0x5eedULL) + uint64_t(ci) * 0x9E3779B97F4A7C15ULL;
        circuits_.push_back(std::move(c));
        plans.push_back(std::move(passes));
    }
    total_amps_ = off;
    // Level-major queue: pass 0 of every circuit, then pass 1, ...
    size_t levels = 0;
    for (auto& p : plans) levels = std::max(levels, p.size());
    uint64_t item = 0;
    for (size_t lv = 0; lv < levels; lv++) {
        for (size_t ci = 0; ci < plans.size(); ci++) {
            if (lv >= plans[ci].size()) continue;
            const TilePass& tp = plans[ci][lv];
            PassRec r;
            std::memset(&r, 0, sizeof r);
            r.state_off = circuits_[ci].state_off;
            r.item_begin = item;
            r.circuit = int(ci);
            r.n = int(circuits_[ci].n);
            r.m = int(tp.qubits.size());
            const uint64_t tiles = uint64_t(1) << (r.n - r.m);
            r.wait_count = uint64_t(lv) * tiles;
            r.op_begin = tp.op_begin;
            r.nops = int(tp.ops.size());
            for (int i = 0; i < r.m; i++) r.q[i] = tp.qubits[i];
            pass_recs_.push_back(r);
            item += tiles;
            tile_bytes_ += 2.0 * (c64_ ? 8.0 : 16.0) * double(uint64_t(1) << r.n);
        }
    }
    total_items_ = item;
    if (max_m_ > 14) fail(kValueError, "tile too large");
    if (max_m_ == 0) max_m_ = 5;  // every circuit runs fused passes: the persistent kernel gets no items

    dev_ = sim.ensure_device();
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cudaStream_t s = dev_->stream;
    const size_t S = c64_ ? 8 : 16;
    const int count = int(circuits_.size());
    amps_.alloc(total_amps_ * S, "batched statevectors");
    recs_.alloc(std::max<size_t>(1, pass_recs_.size()) * sizeof(PassRec), "pass records");
    ops_.alloc(std::max<size_t>(1, ops_host_.size()) * sizeof(TileOp), "tile operations");
    pool_.alloc(std::max<size_t>(1, pool_host_.size()) * sizeof(double2), "gate matrices");
    done_.alloc(std::max(1, count) * 8, "pass counters");
    head_.alloc(16, "work queue head");
    err_.alloc(16, "error flag");
    probs_.alloc(total_amps_ * 8, "probabilities");
    tmp_.alloc(k::scan_tmp_size(total_amps_) * 8 + size_t(count) * 16 + 64, "scan scratch");
    circ_off_.alloc(size_t(count) * 16, "circuit offsets");
    samples_.alloc(std::max<uint64_t>(1, uint64_t(count) * shots_) * 8, "samples");
    zz_part_.alloc(size_t(count) * 8, "expectations");
    seeds_.alloc(size_t(count) * 8, "seeds");
    std::vector<uint64_t> offs(2 * size_t(count)), seeds(count);
    for (int c = 0; c < count; c++) {
        offs[c] = circuits_[c].state_off;
        offs[count + c] = circuits_[c].state_off + (uint64_t(1) << circuits_[c].n);
        seeds[c] = circuits_[c].seed;
    }
    cuda_check(cudaMemcpyAsync(recs_.p, pass_recs_.data(), pass_recs_.size() * sizeof(PassRec), cudaMemcpyHostToDevice, s),
               "upload");
    cuda_check(cudaMemcpyAsync(ops_.p, ops_host_.data(), ops_host_.size() * sizeof(TileOp), cudaMemcpyHostToDevice, s),
               "upload");
    cuda_check(cudaMemcpyAsync(pool_.p, pool_host_.data(), pool_host_.size() * sizeof(double2), cudaMemcpyHostToDevice, s),
               "upload");
    cuda_check(cudaMemcpyAsync(circ_off_.p, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaMemcpyAsync(seeds_.p, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, s), "upload");
    // Fused circuits: executors prepared (pools uploaded, scratch sized) so that
    // runs allocate nothing and can be captured; longest first onto the least
    // loaded side stream.
    std::vector<size_t> order;
    for (size_t ci = 0; ci < circuits_.size(); ci++)
        if (circuits_[ci].fused) order.push_back(ci);
    auto cost = [&](size_t ci) {
        return double(uint64_t(1) << circuits_[ci].n) * double(circuits_[ci].fused->fused_blocks() + 3);
    };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost(a) > cost(b); });
    if (!order.empty()) {
        const size_t nside = std::min<size_t>(kSideStreams, order.size());
        std::vector<double> load(nside, 0.0);
        for (size_t ci : order) {
            const size_t j = size_t(std::min_element(load.begin(), load.end()) - load.begin());
            circuits_[ci].stream = int(j);
            load[j] += cost(ci);
        }
        side_.resize(nside, nullptr);
        join_.resize(nside, nullptr);
        for (size_t j = 0; j < nside; j++) {
            cuda_check(cudaStreamCreateWithFlags(&side_[j], cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaEventCreateWithFlags(&join_[j], cudaEventDisableTiming), "cudaEventCreate");
        }
        cuda_check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "cudaEventCreate");
        for (size_t ci : order) circuits_[ci].fused->prepare(circuit_view(circuits_[ci], s));
    }
    const size_t smem = (S << max_m_);
    // Largest carveout: the occupancy query that sizes the persistent grid must
    // match what the launch gets, since every CTA has to be resident at once.
    if (c64_) {
        cuda_check(cudaFuncSetAttribute(k_batch<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_batch<float2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        int(cudaSharedmemCarveoutMaxShared)),
                   "carveout attribute");
    } else {
        cuda_check(cudaFuncSetAttribute(k_batch<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
                   "smem attribute");
        cuda_check(cudaFuncSetAttribute(k_batch<double2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        int(cudaSharedmemCarveoutMaxShared)),
                   "carveout attribute");
    }
    dev_->sync();
}

BatchRun::~BatchRun() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (dev_) {
        dev_->activate();
        for (cudaStream_t st : side_) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        for (cudaEvent_t e : join_) cudaEventDestroy(e);
        if (fork_) cudaEventDestroy(fork_);
    }
}

k::Batch BatchRun::circuit_view(const Circ& c, cudaStream_t s) const {
    k::Batch b;
    b.stream = s;
    b.c64 = c64_;
    b.amps = static_cast<unsigned char*>(amps_.p) + c.state_off * (c64_ ? 8 : 16);
    b.n = int(c.n);
    b.W = 1;
    b.err = err_.as<int>();
    return b;
}

size_t BatchRun::passes() const {
    size_t total = pass_recs_.size();
    for (const Circ& c : circuits_)
        if (c.fused) total += c.fused->passes();
    return total;
}

size_t BatchRun::fused_circuits() const {
    size_t total = 0;
    for (const Circ& c : circuits_) total += c.fused ? 1 : 0;
    return total;
}

void BatchRun::work(double* bytes, double* tensor_flops, double* cuda_core_flops) const {
    double by = tile_bytes_, tf = 0.0, cf = 0.0;
    for (size_t i = 0; i < pass_recs_.size(); i++) {
        const PassRec& r = pass_recs_[i];
        double per_tile = 0.0;
        for (int k = 0; k < r.nops; k++) {
            const TileOp& op = ops_host_[size_t(r.op_begin + k)];
            const double items = double(uint64_t(1) << (r.m - op.nins));
            switch (op.type) {
                case TileOp::kOne: per_tile += items * 28.0; break;
                case TileOp::kDiagEntry: per_tile += items * 6.0; break;
                case TileOp::kDiagFull: per_tile += double(uint64_t(1) << r.m) * 6.0; break;
                case TileOp::kDense: {
                    const double d = double(1 << op.k);
                    per_tile += double(uint64_t(1) << (r.m - op.k)) * (d * d * 6.0 + (d * d - d) * 2.0);
                    break;
                }
                default: break;
            }
        }
        cf += per_tile * double(uint64_t(1) << (r.n - r.m));
    }
    for (const Circ& c : circuits_) {
        if (!c.fused) continue;
        const k::Batch b = circuit_view(c, nullptr);
        double cc = 0.0, tc = 0.0;
        c.fused->arith_flops(b, &cc, &tc);
        cf += cc;
        tf += tc;
        by += double(c.fused->passes()) * 2.0 * 8.0 * double(uint64_t(1) << c.n);
    }
    *bytes = by;
    *tensor_flops = tf;
    *cuda_core_flops = cf;
}

void BatchRun::enqueue() {
    cudaStream_t s = dev_->stream;
    const size_t S = c64_ ? 8 : 16;
    const int count = int(circuits_.size());
    cuda_check(cudaMemsetAsync(amps_.p, 0, total_amps_ * S, s), "clear states");
    cuda_check(cudaMemsetAsync(done_.p, 0, size_t(count) * 8, s), "clear counters");
    cuda_check(cudaMemsetAsync(head_.p, 0, 16, s), "clear queue");
    cuda_check(cudaMemsetAsync(err_.p, 0, 16, s), "clear error");
    const uint64_t* offs = circ_off_.as<uint64_t>();
    if (c64_)
        k_first_amp<float2><<<(count + 127) / 128, 128, 0, s>>>(amps_.as<float2>(), offs, count);
    else
        k_first_amp<double2><<<(count + 127) / 128, 128, 0, s>>>(amps_.as<double2>(), offs, count);
    if (!side_.empty()) {
        // Fused circuits on the side streams, beside the persistent kernel.
        cuda_check(cudaEventRecord(fork_, s), "fork");
        for (cudaStream_t st : side_) cuda_check(cudaStreamWaitEvent(st, fork_, 0), "fork");
        for (const Circ& c : circuits_)
            if (c.fused) c.fused->run(circuit_view(c, side_[size_t(c.stream)]), nullptr);
        for (size_t j = 0; j < side_.size(); j++) cuda_check(cudaEventRecord(join_[j], side_[j]), "join");
    }
    const size_t smem = (S << max_m_);
    int per_sm = 0;
    if (c64_)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<float2>, kBatchThreads, smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<double2>, kBatchThreads, smem);
    if (per_sm < 1) per_sm = 1;
    // Every CTA is resident at once, so a claimed item never waits on an unclaimed one.
    const unsigned grid = unsigned(std::max<uint64_t>(1, std::min<uint64_t>(total_items_, uint64_t(sm_count()) * per_sm)));
    if (total_items_ > 0) {
        if (c64_)
            k_batch<float2><<<grid, kBatchThreads, smem, s>>>(amps_.as<float2>(), recs_.as<PassRec>(),
                                                             int(pass_recs_.size()), ops_.as<TileOp>(),
                                                             pool_.as<double2>(), done_.as<unsigned long long>(),
                                                             head_.as<unsigned long long>(), total_items_, err_.as<int>());
        else
            k_batch<double2><<<grid, kBatchThreads, smem, s>>>(amps_.as<double2>(), recs_.as<PassRec>(),
                                                              int(pass_recs_.size()), ops_.as<TileOp>(),
                                                              pool_.as<double2>(), done_.as<unsigned long long>(),
                                                              head_.as<unsigned long long>(), total_items_,
                                                              err_.as<int>());
    }
    for (cudaEvent_t e : join_) cuda_check(cudaStreamWaitEvent(s, e, 0), "join");
    const unsigned sgrid = unsigned(std::min<uint64_t>((total_amps_ + 255) / 256, 148 * 32));
    if (c64_)
        k_arena_norm2<float2><<<sgrid, 256, 0, s>>>(amps_.as<float2>(), probs_.as<double>(), total_amps_);
    else
        k_arena_norm2<double2><<<sgrid, 256, 0, s>>>(amps_.as<double2>(), probs_.as<double>(), total_amps_);
    k_zz<<<count, 256, 0, s>>>(probs_.as<double>(), offs, count, zz_part_.as<double>());
    double* tmp = tmp_.as<double>();
    double* base_total = tmp + k::scan_tmp_size(total_amps_);
    k::scan(s, probs_.as<double>(), total_amps_, tmp);
    k_seg_totals<<<(count + 127) / 128, 128, 0, s>>>(probs_.as<double>(), offs, count, base_total, err_.as<int>());
    k_seg_normalize<<<dim3(64, count), 256, 0, s>>>(probs_.as<double>(), offs, count, base_total);
    if (shots_ > 0) {
        const uint64_t th = uint64_t(count) * shots_;
        k_seg_sample<<<unsigned((th + 127) / 128), 128, 0, s>>>(probs_.as<double>(), offs, count, seeds_.as<uint64_t>(),
                                                                shots_, samples_.as<uint64_t>());
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("batch launch: ") + cudaGetErrorString(e));
}

double BatchRun::run(bool use_graph) {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    cudaStream_t s = dev_->stream;
    if (use_graph && !graph_) {
        cudaGraph_t g;
        cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            enqueue();
        } catch (...) {
            cudaStreamEndCapture(s, &g);
            throw;
        }
        cuda_check(cudaStreamEndCapture(s, &g), "end capture");
        cuda_check(cudaGraphInstantiate(&graph_, g, 0), "instantiate graph");
        cudaGraphDestroy(g);
    }
    cudaEvent_t a, b;
    cuda_check(cudaEventCreate(&a), "event");
    cuda_check(cudaEventCreate(&b), "event");
    cuda_check(cudaEventRecord(a, s), "event");
    if (use_graph)
        cuda_check(cudaGraphLaunch(graph_, s), "graph launch");
    else
        enqueue();
    cuda_check(cudaEventRecord(b, s), "event");
    cuda_check(cudaEventSynchronize(b), "event sync");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    int flag = 0;
    cuda_check(cudaMemcpy(&flag, err_.p, 4, cudaMemcpyDeviceToHost), "read error flag");
    if (flag == 1) fail(kRuntimeError, "Invalid state normalization when sampling");
    if (flag == 2) fail(kRuntimeError, "batched pass dependency wait exceeded its limit");
    return double(ms);
}

int BatchRun::error_flag() const {
    int flag = 0;
    cudaMemcpy(&flag, err_.p, 4, cudaMemcpyDeviceToHost);
    return flag;
}

std::unordered_map<std::string, uint64_t> BatchRun::counts(size_t i) const {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    const Circ& c = circuits_.at(i);
    std::vector<uint64_t> h(shots_);
    cuda_check(cudaMemcpy(h.data(), samples_.as<uint64_t>() + i * shots_, shots_ * 8, cudaMemcpyDeviceToHost),
               "read samples");
    std::unordered_map<uint64_t, uint64_t> hist;
    for (auto v : h) hist[v]++;
    std::unordered_map<std::string, uint64_t> out;
    for (auto& kv : hist) {
        std::string key(c.ncb, '0');
        for (auto& cm : c.cbit_map)
            if ((kv.first >> cm.second) & 1) key[c.ncb - 1 - cm.first] = '1';
        out[key] += kv.second;
    }
    return out;
}

std::vector<double> BatchRun::expect_zz() const {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    std::vector<double> v(circuits_.size());
    cuda_check(cudaMemcpy(v.data(), zz_part_.p, v.size() * 8, cudaMemcpyDeviceToHost), "read expectations");
    return v;
}

void BatchRun::statevector(size_t i, double* out) const {
    std::lock_guard<std::mutex> lk(dev_->mu);
    dev_->activate();
    const Circ& c = circuits_.at(i);
    const uint64_t len = uint64_t(1) << c.n;
    if (!c64_) {
        cuda_check(cudaMemcpy(out, amps_.as<double2>() + c.state_off, len * 16, cudaMemcpyDeviceToHost), "read state");
        return;
    }
    std::vector<float> tmp(2 * len);
    cuda_check(cudaMemcpy(tmp.data(), amps_.as<float2>() + c.state_off, len * 8, cudaMemcpyDeviceToHost), "read state");
    for (uint64_t k = 0; k < 2 * len; k++) out[k] = tmp[k];
}

// ---------------------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------------------
TuneResult autotune_tile(Simulator& sim, const std::string& json, bool c64) {
    static std::mutex mu;
    static std::map<std::pair<uint64_t, int>, TuneResult> cache;
    uint64_t n = 0, ncb = 0;
    compile_json(json.data(), json.size(), &n, &ncb);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find({n, c64 ? 1 : 0});
        if (it != cache.end()) return it->second;
    }
    auto time_shape = [&](int m, int fuse, int depth) {
        BatchTuning t;
        t.tile_m = m;
        t.fuse = fuse;
        t.depth = depth;
        BatchRun run(sim, {json}, 0, t);
        run.run(false);
        double ms = 1e30;
        for (int r = 0; r < 3; r++) ms = std::min(ms, run.run(false));
        return ms;
    };
    TuneResult best{c64 ? 13 : 12, 2, 0, 1e30};
    // Tile qubits and fusion width, passes as deep as they grow ...
    const int ms_max = c64 ? 14 : 13;
    for (int m = std::max(5, std::min<int>(10, int(n))); m <= std::min<int>(ms_max, int(n)); m++)
        for (int fuse = 1; fuse <= 3; fuse++) {
            const double ms = time_shape(m, fuse, 0);
            if (ms < best.ms) best = {m, fuse, 0, ms};
        }
    // ... then the shared-memory pass depth of the best shape ...
    for (int depth : {12, 24, 48}) {
        const double ms = time_shape(best.tile_m, best.fuse, depth);
        if (ms < best.ms) best = {best.tile_m, best.fuse, depth, ms};
    }
    // ... and the tensor-core fused passes (complex64, 12 qubits or more).
    if (c64 && n >= uint64_t(kFusedM)) {
        const double ms = time_shape(kFusedM, 5, 0);
        if (ms < best.ms) best = {kFusedM, 5, 0, ms};
    }
    std::lock_guard<std::mutex> lk(mu);
    cache[{n, c64 ? 1 : 0}] = best;
    return best;
}

}  // namespace dq

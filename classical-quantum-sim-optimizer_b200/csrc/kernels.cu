// Per-gate statevector kernels for sm_100a (one HBM pass per operation).
//
// Each kernel restates one loop of src/engine.rs as a flat, coalesced pass:
// a thread owns IPT work items spaced one block-width apart, issues all of its
// 16-byte (c128) or 8-byte (c64) loads before any arithmetic, and touches only
// the amplitudes the operation changes (controls and fixed diagonal patterns
// are folded into the index map, so a CX moves half of the state, a CZ a quarter).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "common.hpp"
#include "kernels.hpp"

namespace dq {
namespace k {
namespace {

using dev::CondList;
using dev::InsertSet;

constexpr int kThreads = 256;
constexpr int kIPT = 4;

inline void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string(what) + ": " + cudaGetErrorString(e));
}

inline unsigned blocks_for(uint64_t items, int per_block) {
    uint64_t b = (items + per_block - 1) / per_block;
    if (b == 0) b = 1;
    if (b > 0x7fffffffULL) fail(kValueError, "launch too large");
    return unsigned(b);
}

InsertSet make_insert(std::vector<int> pos) {
    std::sort(pos.begin(), pos.end());
    if (pos.size() > 8) fail(kValueError, "too many fixed qubits in one operation");
    InsertSet s{};
    s.k = int(pos.size());
    for (size_t i = 0; i < pos.size(); i++) s.pos[i] = pos[i];
    return s;
}

// ---------------------------------------------------------------------------
// 1q gate / X on pairs
// ---------------------------------------------------------------------------
template <typename V>
__global__ void __launch_bounds__(kThreads) k_gate1q(V* __restrict__ s, int n, int nfree, uint64_t items, InsertSet ins,
                                                     uint64_t fixed, uint64_t tbit, double2 u00, double2 u01,
                                                     double2 u10, double2 u11, int is_x, CondList cond,
                                                     const uint64_t* __restrict__ cbits, int cwords) {
    const uint64_t start = uint64_t(blockIdx.x) * (kThreads * kIPT) + threadIdx.x;
    const uint64_t fmask = (uint64_t(1) << nfree) - 1;
    uint64_t idx[kIPT];
    bool act[kIPT];
    V a[kIPT], b[kIPT];
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        uint64_t g = start + uint64_t(t) * kThreads;
        act[t] = g < items;
        idx[t] = 0;
        if (act[t]) {
            uint64_t st = g >> nfree;
            idx[t] = (st << n) | dev::expand(g & fmask, ins) | fixed;
            if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) act[t] = false;
        }
        if (act[t]) {
            a[t] = s[idx[t]];
            b[t] = s[idx[t] + tbit];
        }
    }
    const V m00 = dev::from_d2<V>(u00), m01 = dev::from_d2<V>(u01);
    const V m10 = dev::from_d2<V>(u10), m11 = dev::from_d2<V>(u11);
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        if (!act[t]) continue;
        if (is_x) {
            s[idx[t]] = b[t];
            s[idx[t] + tbit] = a[t];
        } else {
            s[idx[t]] = dev::cadd(dev::cmul(m00, a[t]), dev::cmul(m01, b[t]));
            s[idx[t] + tbit] = dev::cadd(dev::cmul(m10, a[t]), dev::cmul(m11, b[t]));
        }
    }
}

// ---------------------------------------------------------------------------
// SWAP on (01, 10) pairs
// ---------------------------------------------------------------------------
template <typename V>
__global__ void __launch_bounds__(kThreads) k_swap(V* __restrict__ s, int n, int nfree, uint64_t items, InsertSet ins,
                                                   uint64_t fixed, uint64_t lowbit, uint64_t highbit, CondList cond,
                                                   const uint64_t* __restrict__ cbits, int cwords) {
    const uint64_t start = uint64_t(blockIdx.x) * (kThreads * kIPT) + threadIdx.x;
    const uint64_t fmask = (uint64_t(1) << nfree) - 1;
    uint64_t idx[kIPT];
    bool act[kIPT];
    V a[kIPT], b[kIPT];
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        uint64_t g = start + uint64_t(t) * kThreads;
        act[t] = g < items;
        idx[t] = 0;
        if (act[t]) {
            uint64_t st = g >> nfree;
            idx[t] = (st << n) | dev::expand(g & fmask, ins) | fixed;
            if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) act[t] = false;
        }
        if (act[t]) {
            a[t] = s[idx[t] | lowbit];
            b[t] = s[idx[t] | highbit];
        }
    }
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        if (!act[t]) continue;
        s[idx[t] | lowbit] = b[t];
        s[idx[t] | highbit] = a[t];
    }
}

// ---------------------------------------------------------------------------
// Diagonal gates
// ---------------------------------------------------------------------------
struct DiagTable {
    int k;
    int q[5];
    double2 d[32];
};

template <typename V>
__global__ void __launch_bounds__(kThreads) k_diag_full(V* __restrict__ s, int n, uint64_t items, DiagTable tab,
                                                        CondList cond, const uint64_t* __restrict__ cbits, int cwords) {
    const uint64_t start = uint64_t(blockIdx.x) * (kThreads * kIPT) + threadIdx.x;
    const uint64_t lmask = (uint64_t(1) << n) - 1;
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        uint64_t g = start + uint64_t(t) * kThreads;
        if (g >= items) continue;
        if (cond.n && !dev::cond_ok(cond, cbits, cwords, g >> n)) continue;
        uint64_t i = g & lmask;
        int j = 0;
        for (int q = 0; q < tab.k; q++) j = (j << 1) | int((i >> tab.q[q]) & 1);
        s[g] = dev::cmul(s[g], dev::from_d2<V>(tab.d[j]));
    }
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_diag_entry(V* __restrict__ s, int n, int nfree, uint64_t items,
                                                         InsertSet ins, uint64_t fixed, double2 val, CondList cond,
                                                         const uint64_t* __restrict__ cbits, int cwords) {
    const uint64_t start = uint64_t(blockIdx.x) * (kThreads * kIPT) + threadIdx.x;
    const uint64_t fmask = (uint64_t(1) << nfree) - 1;
    const V v = dev::from_d2<V>(val);
    uint64_t idx[kIPT];
    bool act[kIPT];
    V a[kIPT];
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        uint64_t g = start + uint64_t(t) * kThreads;
        act[t] = g < items;
        idx[t] = 0;
        if (act[t]) {
            uint64_t st = g >> nfree;
            idx[t] = (st << n) | dev::expand(g & fmask, ins) | fixed;
            if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) act[t] = false;
        }
        if (act[t]) a[t] = s[idx[t]];
    }
#pragma unroll
    for (int t = 0; t < kIPT; t++)
        if (act[t]) s[idx[t]] = dev::cmul(a[t], v);
}

// ---------------------------------------------------------------------------
// Dense k-qubit gates (k <= 5): gather 2^k amplitudes, multiply, scatter.
// ---------------------------------------------------------------------------
struct Offsets {
    uint64_t o[32];
};

template <typename V, int K>
__global__ void __launch_bounds__(kThreads) k_dense(V* __restrict__ s, int n, int nfree, uint64_t items, InsertSet ins,
                                                    Offsets off, const double2* __restrict__ m, CondList cond,
                                                    const uint64_t* __restrict__ cbits, int cwords) {
    constexpr int D = 1 << K;
    __shared__ double2 sm[D * D];
    for (int i = threadIdx.x; i < D * D; i += blockDim.x) sm[i] = m[i];
    __syncthreads();
    const uint64_t g = uint64_t(blockIdx.x) * kThreads + threadIdx.x;
    if (g >= items) return;
    const uint64_t st = g >> nfree;
    if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) return;
    const uint64_t base = (st << n) | dev::expand(g & ((uint64_t(1) << nfree) - 1), ins);
    V v[D];
#pragma unroll
    for (int j = 0; j < D; j++) v[j] = s[base | off.o[j]];
#pragma unroll 1
    for (int row = 0; row < D; row++) {
        V acc = dev::czero<V>();
#pragma unroll
        for (int col = 0; col < D; col++) acc = dev::cadd(acc, dev::cmul(dev::from_d2<V>(sm[row * D + col]), v[col]));
        s[base | off.o[row]] = acc;
    }
}

// ---------------------------------------------------------------------------
// Measurement: branch sums, per-state draw, collapse
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of two values; result valid in thread 0.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
    __shared__ double sa[32], sb[32];
    a = warp_sum(a);
    b = warp_sum(b);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_prob2(const V* __restrict__ s, int n, int chunk_bits, int P, uint64_t qbit,
                                                    double* __restrict__ partial, CondList cond,
                                                    const uint64_t* __restrict__ cbits, int cwords) {
    const uint64_t st = blockIdx.x / P;
    const uint64_t c = blockIdx.x % P;
    if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) return;
    const uint64_t off = c << chunk_bits;
    const uint64_t base = (st << n) + off;
    const uint64_t len = uint64_t(1) << chunk_bits;
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) {
        double v = dev::norm2(s[base + i]);
        if ((off + i) & qbit)
            p1 += v;
        else
            p0 += v;
    }
    block_sum2(p0, p1);
    if (threadIdx.x == 0) {
        partial[(st * P + c) * 2] = p0;
        partial[(st * P + c) * 2 + 1] = p1;
    }
}

__global__ void k_measure_finalize(uint64_t W, int P, const double* __restrict__ partial,
                                   const uint64_t* __restrict__ rng_seed, uint64_t* __restrict__ draws,
                                   int* __restrict__ outcome, double* __restrict__ scale, uint64_t* __restrict__ cbits,
                                   int cwords, int64_t cbit, CondList cond, int* __restrict__ err) {
    const uint64_t st = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (st >= W) return;
    if (cond.n && !dev::cond_ok(cond, cbits, cwords, st)) {
        outcome[st] = -1;
        return;
    }
    double p0 = 0.0, p1 = 0.0;
    for (int c = 0; c < P; c++) {
        p0 += partial[(st * P + c) * 2];
        p1 += partial[(st * P + c) * 2 + 1];
    }
    double total = p0 + p1;
    if (!(isfinite(total) && total > 0.0)) {
        *err = 1;
        outcome[st] = -1;
        return;
    }
    uint64_t k = draws[st];
    draws[st] = k + 1;
    double r = dev::u64_to_unit(dev::chacha8_u64(rng_seed[st], k));
    int o = r < p1 / total ? 1 : 0;
    outcome[st] = o;
    scale[st] = 1.0 / sqrt(o ? p1 : p0);
    if (cbit >= 0) {
        uint64_t* w = cbits + st * uint64_t(cwords) + (uint64_t(cbit) >> 6);
        uint64_t bit = uint64_t(1) << (uint64_t(cbit) & 63);
        *w = o ? (*w | bit) : (*w & ~bit);
    }
}

template <typename V>
__global__ void __launch_bounds__(kThreads) k_collapse(V* __restrict__ s, int n, uint64_t items, int q,
                                                       const int* __restrict__ outcome,
                                                       const double* __restrict__ scale, int reset) {
    const uint64_t start = uint64_t(blockIdx.x) * (kThreads * kIPT) + threadIdx.x;
    const int nf = n - 1;
    const uint64_t fmask = (uint64_t(1) << nf) - 1;
    const uint64_t qb = uint64_t(1) << q;
#pragma unroll
    for (int t = 0; t < kIPT; t++) {
        uint64_t g = start + uint64_t(t) * kThreads;
        if (g >= items) continue;
        uint64_t st = g >> nf;
        int o = outcome[st];
        if (o < 0) continue;
        double sc = scale[st];
        uint64_t j = g & fmask;
        uint64_t low = qb - 1;
        uint64_t i0 = (st << n) | (j & low) | ((j & ~low) << 1);
        uint64_t i1 = i0 | qb;
        if (o == 0) {
            s[i0] = dev::cscale(s[i0], sc);
            s[i1] = dev::czero<V>();
        } else if (reset) {
            s[i0] = dev::cscale(s[i1], sc);
            s[i1] = dev::czero<V>();
        } else {
            s[i0] = dev::czero<V>();
            s[i1] = dev::cscale(s[i1], sc);
        }
    }
}

// ---------------------------------------------------------------------------
// State initialisation
// ---------------------------------------------------------------------------
template <typename V>
__global__ void k_set_first(V* s, int n, uint64_t W) {
    uint64_t st = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (st < W) {
        V one = dev::czero<V>();
        one.x = 1;
        s[st << n] = one;
    }
}

template <typename V>
__global__ void k_broadcast(V* __restrict__ dst, const V* __restrict__ src, int n, uint64_t items) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < items; g += uint64_t(gridDim.x) * blockDim.x)
        dst[g] = src[g & ((uint64_t(1) << n) - 1)];
}

// ---------------------------------------------------------------------------
// Probabilities, CDF, sampling
// ---------------------------------------------------------------------------
template <typename V>
__global__ void k_norm2(const V* __restrict__ s, double* __restrict__ out, uint64_t len) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x)
        out[g] = dev::norm2(s[g]);
}

struct QSel {
    int k;
    int q[64];
};

// Parallel bit deposit: the low bits of x go to the set bits of mask, in order.
__device__ __forceinline__ uint64_t pdep(uint64_t x, uint64_t mask) {
    uint64_t out = 0;
    while (mask) {
        uint64_t low = mask & (~mask + 1);
        if (x & 1) out |= low;
        x >>= 1;
        mask ^= low;
    }
    return out;
}

// out[j] = sum over the unselected bits r of |s[pdep(r, rest) | deposit(j)]|^2,
// G threads per output summing r = lane, lane+G, ... then a fixed-order tree,
// so the result does not depend on scheduling.
template <typename V>
__global__ void __launch_bounds__(256) k_marginal(const V* __restrict__ s, int n, QSel sel, uint64_t rest_mask,
                                                 int G_bits, double* __restrict__ out, uint64_t nout) {
    __shared__ double sm[256];
    const int G = 1 << G_bits;
    const int lane = threadIdx.x & (G - 1);
    const uint64_t j = (uint64_t(blockIdx.x) * 256 + threadIdx.x) >> G_bits;
    double acc = 0.0;
    if (j < nout) {
        uint64_t base = 0;
        for (int t = 0; t < sel.k; t++) base |= ((j >> (sel.k - 1 - t)) & 1) << sel.q[t];
        const uint64_t terms = uint64_t(1) << (n - sel.k);
        for (uint64_t r = lane; r < terms; r += G) acc += dev::norm2(s[base | pdep(r, rest_mask)]);
    }
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int w = G >> 1; w > 0; w >>= 1) {
        if (lane < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (lane == 0 && j < nout) out[j] = sm[threadIdx.x];
}

constexpr int kScanItems = 8;
constexpr int kScanTile = 256 * kScanItems;

// Tile-local inclusive scan of `in` into x (V = double: in == x, in place;
// V = float2 / double2: the squared magnitudes of a state, as k_norm2 computes
// them, so the probability table is never written and re-read).
template <typename V>
__global__ void __launch_bounds__(256) k_scan_tiles(const V* __restrict__ in, double* __restrict__ x, uint64_t len,
                                                    double* __restrict__ sums) {
    __shared__ double warp_tot[8];
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    double v[kScanItems];
    double run = 0.0;
    // A whole run of complex64 amplitudes is read as 16-byte vectors (two
    // amplitudes each); the sums are the same, in the same order.
    const bool full = base + kScanItems <= len;
    bool done = false;
    if constexpr (std::is_same<V, float2>::value) {
        if (full && (reinterpret_cast<uintptr_t>(in) & 15) == 0) {
            const float4* p = reinterpret_cast<const float4*>(in + base);
            float4 f[kScanItems / 2];
#pragma unroll
            for (int i = 0; i < kScanItems / 2; i++) f[i] = p[i];
#pragma unroll
            for (int i = 0; i < kScanItems / 2; i++) {
                run += dev::norm2(make_float2(f[i].x, f[i].y));
                v[2 * i] = run;
                run += dev::norm2(make_float2(f[i].z, f[i].w));
                v[2 * i + 1] = run;
            }
            done = true;
        }
    }
    if (!done) {
#pragma unroll
        for (int i = 0; i < kScanItems; i++) {
            double e = 0.0;
            if (base + i < len) {
                if constexpr (std::is_same<V, double>::value)
                    e = in[base + i];
                else
                    e = dev::norm2(in[base + i]);
            }
            run += e;
            v[i] = run;
        }
    }
    // inclusive warp scan of thread totals
    double t = run;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
    }
    if (lane == 31) warp_tot[w] = t;
    __syncthreads();
    double wprefix = 0.0;
    for (int i = 0; i < w; i++) wprefix += warp_tot[i];
    double excl = wprefix + t - run;
    if (full && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
        double2* px = reinterpret_cast<double2*>(x + base);
#pragma unroll
        for (int i = 0; i < kScanItems / 2; i++) px[i] = make_double2(v[2 * i] + excl, v[2 * i + 1] + excl);
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; i++)
            if (base + i < len) x[base + i] = v[i] + excl;
    }
    if (threadIdx.x == 255) {
        double tot = 0.0;
        for (int i = 0; i < 8; i++) tot += warp_tot[i];
        sums[blockIdx.x] = tot;
    }
}

__global__ void k_scan_add(double* __restrict__ x, uint64_t len, const double* __restrict__ sums) {
    const uint64_t blk = blockIdx.x + 1;  // tile 0 needs no offset
    const double add = sums[blk - 1];
    for (uint64_t i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        uint64_t g = blk * kScanTile + i;
        if (g < len) x[g] += add;
    }
}

__global__ void k_cdf_normalize(double* __restrict__ cdf, uint64_t len, double total, int clamp) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x) {
        double v = cdf[g] / total;
        if (clamp) v = fmin(v, 1.0);
        cdf[g] = (g == len - 1) ? 1.0 : v;
    }
}

// Entry i of running sums kept in two levels: tile-local sums x plus the
// inclusive sums of whole tiles before it (the same addition k_scan_add makes).
__device__ __forceinline__ double two_level(const double* __restrict__ x, const double* __restrict__ tiles,
                                            uint64_t i) {
    double v = x[i];
    if (tiles && i >= uint64_t(kScanTile)) v = v + tiles[i / uint64_t(kScanTile) - 1];
    return v;
}

__global__ void k_take_total(const double* __restrict__ cdf, uint64_t len, const double* __restrict__ tiles,
                             double* scalar, int* err) {
    double t = two_level(cdf, tiles, len - 1);
    *scalar = t;
    if (!(isfinite(t) && t > 0.0)) *err = 1;
}

__global__ void k_cdf_normalize_dev(double* __restrict__ cdf, uint64_t len, const double* __restrict__ scalar,
                                    int clamp) {
    const double total = *scalar;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x) {
        double v = cdf[g] / total;
        if (clamp) v = fmin(v, 1.0);
        cdf[g] = (g == len - 1) ? 1.0 : v;
    }
}

// With `total` (device scalar, or host value when total_dev is null and
// total_host > 0) the table holds the unnormalised running sums and each
// probe normalises the entry it reads exactly as k_cdf_normalize would have
// stored it (cdf[i] / total, clamped to 1 when clamp, the last entry 1).
__global__ void k_sample(const double* __restrict__ cdf, uint64_t len, uint64_t seed, uint64_t shots, int per_shot,
                         const double* __restrict__ tiles, const double* __restrict__ total_dev, double total_host,
                         int clamp, uint64_t* __restrict__ out) {
    uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= shots) return;
    const bool scaled = total_dev != nullptr || total_host > 0.0;
    const double total = total_dev ? *total_dev : total_host;
    uint64_t v = per_shot ? dev::chacha8_u64(seed + t, 0) : dev::chacha8_u64(seed, t);
    double draw = dev::u64_to_unit(v);
    uint64_t lo = 0, hi = len;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        double c = two_level(cdf, tiles, mid);
        if (scaled) {
            c = c / total;
            if (clamp) c = fmin(c, 1.0);
            if (mid == len - 1) c = 1.0;
        }
        if (c <= draw)
            lo = mid + 1;
        else
            hi = mid;
    }
    out[t] = lo < len - 1 ? lo : len - 1;
}

template <typename V>
__global__ void __launch_bounds__(256) k_dot(const V* __restrict__ a, const double2* __restrict__ b, uint64_t len,
                                            double2* __restrict__ partial) {
    double re = 0.0, im = 0.0;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x) {
        V x = a[g];
        double2 y = b[g];
        double xr = x.x, xi = -double(x.y);
        re += xr * y.x - xi * y.y;
        im += xr * y.y + xi * y.x;
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(re, im);
}

template <typename VA, typename VB>
__global__ void __launch_bounds__(256) k_compare(const VA* __restrict__ a, const VB* __restrict__ b, uint64_t len,
                                                double* __restrict__ partial) {
    double re = 0.0, im = 0.0, mx = 0.0, na = 0.0, nb = 0.0;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x) {
        VA x = a[g];
        VB y = b[g];
        double xr = x.x, xi = x.y, yr = y.x, yi = y.y;
        re += xr * yr + xi * yi;
        im += xr * yi - xi * yr;
        na += xr * xr + xi * xi;
        nb += yr * yr + yi * yi;
        double dr = xr - yr, di = xi - yi;
        mx = fmax(mx, sqrt(dr * dr + di * di));
    }
    block_sum2(re, im);
    __syncthreads();  // block_sum2's shared partials are reused below
    block_sum2(na, nb);
    __shared__ double smx[32];
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smx[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); w++) m = fmax(m, smx[w]);
        partial[blockIdx.x * 5] = re;
        partial[blockIdx.x * 5 + 1] = im;
        partial[blockIdx.x * 5 + 2] = m;
        partial[blockIdx.x * 5 + 3] = na;
        partial[blockIdx.x * 5 + 4] = nb;
    }
}

template <typename V>
__global__ void k_gather(const V* __restrict__ s, const uint64_t* __restrict__ idx, uint64_t count,
                         double2* __restrict__ out) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < count; g += uint64_t(gridDim.x) * blockDim.x) {
        const V v = s[idx[g]];
        out[g] = make_double2(v.x, v.y);
    }
}

// Partials of sum_i (-1)^popcount((i ^ x) & z) conj(a_i) a_(i ^ x): <a|X^x Z^z|a>.
template <typename V>
__global__ void __launch_bounds__(256) k_pauli(const V* __restrict__ a, uint64_t len, uint64_t x, uint64_t z,
                                              double2* __restrict__ partial) {
    double re = 0.0, im = 0.0;
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x) {
        const V u = a[g];
        const V w = a[g ^ x];
        const double sgn = (__popcll((g ^ x) & z) & 1) ? -1.0 : 1.0;
        const double ur = u.x, ui = -double(u.y);
        re += sgn * (ur * w.x - ui * w.y);
        im += sgn * (ur * w.y + ui * w.x);
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(re, im);
}

__global__ void k_widen(const float2* __restrict__ s, double2* __restrict__ out, uint64_t len) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x)
        out[g] = make_double2(s[g].x, s[g].y);
}

uint64_t control_fixed(const std::vector<Ctl>& controls) {
    uint64_t v = 0;
    for (auto& c : controls)
        if (c.value) v |= uint64_t(1) << c.qubit;
    return v;
}

template <typename V>
void gate1q_t(const Batch& b, int target, const std::vector<Ctl>& controls, const double2 u[4], bool is_x,
              const CondList& cond) {
    std::vector<int> pos{target};
    for (auto& c : controls) pos.push_back(c.qubit);
    InsertSet ins = make_insert(pos);
    int nfree = b.n - ins.k;
    uint64_t items = b.W << nfree;
    k_gate1q<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(
        static_cast<V*>(b.amps), b.n, nfree, items, ins, control_fixed(controls), uint64_t(1) << target, u[0], u[1],
        u[2], u[3], is_x ? 1 : 0, cond, b.cbits, b.cwords);
    check_launch("gate1q");
}

template <typename V>
void swap_t(const Batch& b, int qa, int qb, const std::vector<Ctl>& controls, const CondList& cond) {
    std::vector<int> pos{qa, qb};
    for (auto& c : controls) pos.push_back(c.qubit);
    InsertSet ins = make_insert(pos);
    int nfree = b.n - ins.k;
    uint64_t items = b.W << nfree;
    int lo = std::min(qa, qb), hi = std::max(qa, qb);
    k_swap<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(
        static_cast<V*>(b.amps), b.n, nfree, items, ins, control_fixed(controls), uint64_t(1) << lo, uint64_t(1) << hi,
        cond, b.cbits, b.cwords);
    check_launch("swap");
}

template <typename V>
void diagonal_t(const Batch& b, const std::vector<int>& qubits, const std::vector<double2>& diag,
                const CondList& cond) {
    const int kq = int(qubits.size());
    std::vector<int> nontrivial;
    for (int j = 0; j < (1 << kq); j++)
        if (!(diag[j].x == 1.0 && diag[j].y == 0.0)) nontrivial.push_back(j);
    if (nontrivial.empty()) return;
    if (int(nontrivial.size()) * 2 <= (1 << kq)) {
        InsertSet ins = make_insert(qubits);
        int nfree = b.n - kq;
        uint64_t items = b.W << nfree;
        for (int j : nontrivial) {
            uint64_t fixed = 0;
            for (int t = 0; t < kq; t++)
                if ((j >> (kq - 1 - t)) & 1) fixed |= uint64_t(1) << qubits[t];
            k_diag_entry<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(
                static_cast<V*>(b.amps), b.n, nfree, items, ins, fixed, diag[j], cond, b.cbits, b.cwords);
            check_launch("diag_entry");
        }
        return;
    }
    DiagTable tab{};
    tab.k = kq;
    for (int t = 0; t < kq; t++) tab.q[t] = qubits[t];
    for (int j = 0; j < (1 << kq); j++) tab.d[j] = diag[j];
    uint64_t items = b.W << b.n;
    k_diag_full<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(static_cast<V*>(b.amps), b.n, items,
                                                                                   tab, cond, b.cbits, b.cwords);
    check_launch("diag_full");
}

template <typename V, int K>
void dense_k(const Batch& b, const std::vector<int>& qubits, const double2* dm, const CondList& cond) {
    Offsets off{};
    for (int j = 0; j < (1 << K); j++) {
        uint64_t o = 0;
        for (int bit = 0; bit < K; bit++) o |= uint64_t((j >> (K - 1 - bit)) & 1) << qubits[bit];
        off.o[j] = o;
    }
    InsertSet ins = make_insert(qubits);
    int nfree = b.n - K;
    uint64_t items = b.W << nfree;
    k_dense<V, K><<<blocks_for(items, kThreads), kThreads, 0, b.stream>>>(static_cast<V*>(b.amps), b.n, nfree, items,
                                                                          ins, off, dm, cond, b.cbits, b.cwords);
    check_launch("dense");
}

template <typename V>
void dense_t(const Batch& b, const std::vector<int>& qubits, const double2* dm, const CondList& cond) {
    switch (qubits.size()) {
        case 1: dense_k<V, 1>(b, qubits, dm, cond); break;
        case 2: dense_k<V, 2>(b, qubits, dm, cond); break;
        case 3: dense_k<V, 3>(b, qubits, dm, cond); break;
        case 4: dense_k<V, 4>(b, qubits, dm, cond); break;
        case 5: dense_k<V, 5>(b, qubits, dm, cond); break;
        default: fail(kValueError, "Dense gate arity exceeds supported maximum");
    }
}

template <typename V>
void measure_t(const Batch& b, int qubit, int64_t cbit, bool reset, const CondList& cond) {
    int pbits = std::max(0, std::min(10, b.n - 12));
    int P = 1 << pbits;
    int chunk_bits = b.n - pbits;
    uint64_t grid = b.W * uint64_t(P);
    k_prob2<V><<<blocks_for(grid, 1), kThreads, 0, b.stream>>>(static_cast<const V*>(b.amps), b.n, chunk_bits, P,
                                                              uint64_t(1) << qubit, b.partial, cond, b.cbits, b.cwords);
    check_launch("prob2");
    k_measure_finalize<<<blocks_for(b.W, 128), 128, 0, b.stream>>>(b.W, P, b.partial, b.rng_seed, b.draws, b.outcome,
                                                                  b.scale, b.cbits, b.cwords, cbit, cond, b.err);
    check_launch("measure_finalize");
    uint64_t items = b.W << (b.n - 1);
    k_collapse<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(
        static_cast<V*>(b.amps), b.n, items, qubit, b.outcome, b.scale, reset ? 1 : 0);
    check_launch("collapse");
}

template <typename V>
void measure_draw_t(const Batch& b, int qubit, double draw, int* outcome_host) {
    const int pbits = std::max(0, std::min(10, b.n - 12));
    const int P = 1 << pbits;
    k_prob2<V><<<P, kThreads, 0, b.stream>>>(static_cast<const V*>(b.amps), b.n, b.n - pbits, P, uint64_t(1) << qubit,
                                            b.partial, CondList{}, b.cbits, b.cwords);
    check_launch("prob2");
    std::vector<double> part(size_t(P) * 2);
    cudaError_t e = cudaMemcpyAsync(part.data(), b.partial, part.size() * 8, cudaMemcpyDeviceToHost, b.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b.stream);
    if (e != cudaSuccess) fail(kCudaError, std::string("branch sums: ") + cudaGetErrorString(e));
    // The branch sums in the order k_measure_finalize adds them.
    double p0 = 0.0, p1 = 0.0;
    for (int c = 0; c < P; c++) {
        p0 += part[size_t(c) * 2];
        p1 += part[size_t(c) * 2 + 1];
    }
    const double total = p0 + p1;
    if (!(std::isfinite(total) && total > 0.0)) fail(kRuntimeError, "Cannot measure a state with nonfinite or zero norm");
    const int o = draw < p1 / total ? 1 : 0;  // engine.rs:405
    const double scale = 1.0 / std::sqrt(o ? p1 : p0);
    e = cudaMemcpyAsync(b.outcome, &o, sizeof(int), cudaMemcpyHostToDevice, b.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.scale, &scale, sizeof(double), cudaMemcpyHostToDevice, b.stream);
    if (e != cudaSuccess) fail(kCudaError, std::string("measurement upload: ") + cudaGetErrorString(e));
    const uint64_t items = uint64_t(1) << (b.n - 1);
    k_collapse<V><<<blocks_for(items, kThreads * kIPT), kThreads, 0, b.stream>>>(static_cast<V*>(b.amps), b.n, items,
                                                                                  qubit, b.outcome, b.scale, 0);
    check_launch("collapse");
    // The host values above must not change before the copies read them.
    e = cudaStreamSynchronize(b.stream);
    if (e != cudaSuccess) fail(kCudaError, std::string("collapse: ") + cudaGetErrorString(e));
    *outcome_host = o;
}

// out[i * 2^nl + j] = left[j] * right[i]: the state of the merged block whose
// low nl qubits are the left block's (src/distributed/pblock/model.rs:216-230).
template <typename V>
__global__ void k_kron(const V* __restrict__ left, int nl, const V* __restrict__ right, uint64_t len,
                       V* __restrict__ out) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < len; g += uint64_t(gridDim.x) * blockDim.x)
        out[g] = dev::cmul(left[g & ((uint64_t(1) << nl) - 1)], right[g >> nl]);
}

unsigned stream_grid(uint64_t len) {
    uint64_t b = (len + 255) / 256;
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(b, 148 * 32)));
}

}  // namespace

void gate1q(const Batch& b, int target, const std::vector<Ctl>& controls, const double2 u[4], bool is_x,
            const CondList& cond) {
    if (b.c64)
        gate1q_t<float2>(b, target, controls, u, is_x, cond);
    else
        gate1q_t<double2>(b, target, controls, u, is_x, cond);
}

void swap(const Batch& b, int qa, int qb, const std::vector<Ctl>& controls, const CondList& cond) {
    if (b.c64)
        swap_t<float2>(b, qa, qb, controls, cond);
    else
        swap_t<double2>(b, qa, qb, controls, cond);
}

void diagonal(const Batch& b, const std::vector<int>& qubits, const std::vector<double2>& diag, const CondList& cond) {
    if (b.c64)
        diagonal_t<float2>(b, qubits, diag, cond);
    else
        diagonal_t<double2>(b, qubits, diag, cond);
}

void dense(const Batch& b, const std::vector<int>& qubits, const double2* dm, const CondList& cond) {
    if (b.c64)
        dense_t<float2>(b, qubits, dm, cond);
    else
        dense_t<double2>(b, qubits, dm, cond);
}

void measure(const Batch& b, int qubit, int64_t cbit, bool reset, const CondList& cond) {
    if (b.c64)
        measure_t<float2>(b, qubit, cbit, reset, cond);
    else
        measure_t<double2>(b, qubit, cbit, reset, cond);
}

void measure_draw(const Batch& b, int qubit, double draw, int* outcome) {
    if (b.W != 1) fail(kValueError, "a measurement with a given draw takes one state");
    if (b.c64)
        measure_draw_t<float2>(b, qubit, draw, outcome);
    else
        measure_draw_t<double2>(b, qubit, draw, outcome);
}

void kron(cudaStream_t s, bool c64, const void* left, int nl, const void* right, int nr, void* out) {
    const uint64_t len = uint64_t(1) << (nl + nr);
    if (c64)
        k_kron<float2><<<stream_grid(len), 256, 0, s>>>(static_cast<const float2*>(left), nl,
                                                         static_cast<const float2*>(right), len, static_cast<float2*>(out));
    else
        k_kron<double2><<<stream_grid(len), 256, 0, s>>>(static_cast<const double2*>(left), nl,
                                                          static_cast<const double2*>(right), len,
                                                          static_cast<double2*>(out));
    check_launch("kron");
}

void init_basis(const Batch& b) {
    size_t bytes = size_t(b.W << b.n) * (b.c64 ? 8 : 16);
    cudaMemsetAsync(b.amps, 0, bytes, b.stream);
    if (b.c64)
        k_set_first<float2><<<blocks_for(b.W, 128), 128, 0, b.stream>>>(static_cast<float2*>(b.amps), b.n, b.W);
    else
        k_set_first<double2><<<blocks_for(b.W, 128), 128, 0, b.stream>>>(static_cast<double2*>(b.amps), b.n, b.W);
    check_launch("init_basis");
}

void broadcast(const Batch& b, const void* src) {
    uint64_t items = b.W << b.n;
    if (b.c64)
        k_broadcast<float2><<<stream_grid(items), 256, 0, b.stream>>>(static_cast<float2*>(b.amps),
                                                                       static_cast<const float2*>(src), b.n, items);
    else
        k_broadcast<double2><<<stream_grid(items), 256, 0, b.stream>>>(static_cast<double2*>(b.amps),
                                                                        static_cast<const double2*>(src), b.n, items);
    check_launch("broadcast");
}

void norm2(const Batch& b, double* out) {
    uint64_t len = uint64_t(1) << b.n;
    if (b.c64)
        k_norm2<float2><<<stream_grid(len), 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), out, len);
    else
        k_norm2<double2><<<stream_grid(len), 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), out, len);
    check_launch("norm2");
}

void marginal(const Batch& b, const std::vector<int>& qubits, double* out) {
    QSel sel{};
    sel.k = int(qubits.size());
    uint64_t sel_mask = 0;
    for (int t = 0; t < sel.k; t++) {
        sel.q[t] = qubits[t];
        sel_mask |= uint64_t(1) << qubits[t];
    }
    uint64_t full = b.n >= 64 ? ~uint64_t(0) : (uint64_t(1) << b.n) - 1;
    uint64_t rest_mask = full & ~sel_mask;
    int rest = b.n - sel.k;
    uint64_t nout = uint64_t(1) << sel.k;
    int G_bits = 0;
    // About 2^20 threads in flight, at most 256 per output.
    while (G_bits < 8 && G_bits < rest && (nout << (G_bits + 1)) <= (uint64_t(1) << 20)) G_bits++;
    uint64_t threads = nout << G_bits;
    unsigned grid = blocks_for(threads, 256);
    if (b.c64)
        k_marginal<float2><<<grid, 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), b.n, sel, rest_mask, G_bits,
                                                       out, nout);
    else
        k_marginal<double2><<<grid, 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), b.n, sel, rest_mask,
                                                        G_bits, out, nout);
    check_launch("marginal");
}

size_t scan_tmp_size(uint64_t len) {
    size_t total = 0;
    while (len > uint64_t(kScanTile)) {
        len = (len + kScanTile - 1) / kScanTile;
        total += len;
    }
    return total + 1;
}

int scan_launches(uint64_t len) {
    const uint64_t nb = (len + kScanTile - 1) / kScanTile;
    return nb > 1 ? 2 + scan_launches(nb) : 1;
}

void scan(cudaStream_t s, double* x, uint64_t len, double* tmp) {
    uint64_t nb = (len + kScanTile - 1) / kScanTile;
    k_scan_tiles<double><<<blocks_for(nb, 1), 256, 0, s>>>(x, x, len, tmp);
    check_launch("scan_tiles");
    if (nb > 1) {
        scan(s, tmp, nb, tmp + nb);
        k_scan_add<<<blocks_for(nb - 1, 1), 256, 0, s>>>(x, len, tmp);
        check_launch("scan_add");
    }
}

void scan_probs(const Batch& b, double* x, double* tmp, bool add_tiles) {
    const uint64_t len = uint64_t(1) << b.n;
    const uint64_t nb = (len + kScanTile - 1) / kScanTile;
    if (b.c64)
        k_scan_tiles<float2><<<blocks_for(nb, 1), 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), x, len, tmp);
    else
        k_scan_tiles<double2>
            <<<blocks_for(nb, 1), 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), x, len, tmp);
    check_launch("scan_probs");
    if (nb > 1) {
        scan(b.stream, tmp, nb, tmp + nb);
        if (add_tiles) {
            k_scan_add<<<blocks_for(nb - 1, 1), 256, 0, b.stream>>>(x, len, tmp);
            check_launch("scan_add");
        }
    }
}

void scan_local(cudaStream_t s, double* x, uint64_t len, double* tmp) {
    uint64_t nb = (len + kScanTile - 1) / kScanTile;
    k_scan_tiles<double><<<blocks_for(nb, 1), 256, 0, s>>>(x, x, len, tmp);
    check_launch("scan_tiles");
    if (nb > 1) scan(s, tmp, nb, tmp + nb);
}

uint64_t scan_tile_of(uint64_t i) { return i / uint64_t(kScanTile); }

void take_total(cudaStream_t s, const double* cdf, uint64_t len, const double* tiles, double* scalar, int* err) {
    k_take_total<<<1, 1, 0, s>>>(cdf, len, tiles, scalar, err);
    check_launch("take_total");
}

void cdf_normalize(cudaStream_t s, double* cdf, uint64_t len, double total, bool clamp) {
    k_cdf_normalize<<<stream_grid(len), 256, 0, s>>>(cdf, len, total, clamp ? 1 : 0);
    check_launch("cdf_normalize");
}

void cdf_normalize_device(cudaStream_t s, double* cdf, uint64_t len, double* scalar, int* err, bool clamp) {
    k_take_total<<<1, 1, 0, s>>>(cdf, len, nullptr, scalar, err);
    k_cdf_normalize_dev<<<stream_grid(len), 256, 0, s>>>(cdf, len, scalar, clamp ? 1 : 0);
    check_launch("cdf_normalize_device");
}

void sample(cudaStream_t s, const double* cdf, uint64_t len, uint64_t seed, uint64_t shots, bool per_shot_seed,
            uint64_t* out) {
    if (shots == 0) return;
    k_sample<<<blocks_for(shots, 128), 128, 0, s>>>(cdf, len, seed, shots, per_shot_seed ? 1 : 0, nullptr, nullptr,
                                                     0.0, 0, out);
    check_launch("sample");
}

void sample_sums(cudaStream_t s, const double* sums, const double* tiles, uint64_t len, const double* total_dev,
                 double total_host, bool clamp, uint64_t seed, uint64_t shots, bool per_shot_seed, uint64_t* out) {
    if (shots == 0) return;
    k_sample<<<blocks_for(shots, 128), 128, 0, s>>>(sums, len, seed, shots, per_shot_seed ? 1 : 0, tiles, total_dev,
                                                     total_host, clamp ? 1 : 0, out);
    check_launch("sample");
}

int dot_partials(const Batch& b, const double2* other, double2* partial) {
    uint64_t len = uint64_t(1) << b.n;
    if (b.c64)
        k_dot<float2><<<kDotBlocks, 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), other, len, partial);
    else
        k_dot<double2><<<kDotBlocks, 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), other, len, partial);
    check_launch("dot");
    return kDotBlocks;
}

void gather(const Batch& b, const uint64_t* idx, uint64_t count, double2* out) {
    if (count == 0) return;
    const unsigned grid = unsigned(std::min<uint64_t>((count + 255) / 256, 1184));
    if (b.c64)
        k_gather<float2><<<grid, 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), idx, count, out);
    else
        k_gather<double2><<<grid, 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), idx, count, out);
    check_launch("gather");
}

int pauli_partials(const Batch& b, uint64_t x, uint64_t z, double2* partial) {
    const uint64_t len = uint64_t(1) << b.n;
    if (b.c64)
        k_pauli<float2><<<kDotBlocks, 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), len, x, z, partial);
    else
        k_pauli<double2><<<kDotBlocks, 256, 0, b.stream>>>(static_cast<const double2*>(b.amps), len, x, z, partial);
    check_launch("pauli expectation");
    return kDotBlocks;
}

void compare(cudaStream_t s, const void* a, bool a64, const void* b, bool b64, uint64_t len, double* partial) {
    if (!a64 && !b64)
        k_compare<double2, double2><<<kDotBlocks, 256, 0, s>>>(static_cast<const double2*>(a),
                                                               static_cast<const double2*>(b), len, partial);
    else if (!a64 && b64)
        k_compare<double2, float2><<<kDotBlocks, 256, 0, s>>>(static_cast<const double2*>(a),
                                                              static_cast<const float2*>(b), len, partial);
    else if (a64 && !b64)
        k_compare<float2, double2><<<kDotBlocks, 256, 0, s>>>(static_cast<const float2*>(a),
                                                              static_cast<const double2*>(b), len, partial);
    else
        k_compare<float2, float2><<<kDotBlocks, 256, 0, s>>>(static_cast<const float2*>(a),
                                                             static_cast<const float2*>(b), len, partial);
    check_launch("compare");
}

void widen(const Batch& b, double2* out) {
    uint64_t len = uint64_t(1) << b.n;
    k_widen<<<stream_grid(len), 256, 0, b.stream>>>(static_cast<const float2*>(b.amps), out, len);
    check_launch("widen");
}

}  // namespace k
}  // namespace dq

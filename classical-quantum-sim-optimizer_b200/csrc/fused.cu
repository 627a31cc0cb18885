// Fused 5-qubit blocks as tcgen05 tensor-core contractions (complex64 state).
//
// A CTA owns one 2^12-amplitude tile at a time.  For block j (a 32x32 complex
// matrix U on 5 tile qubits) the tile is held in shared memory as the A
// operand of D = A * B: 128 rows (the tile's 128 "columns", i.e. values of the
// other 7 tile qubits) by K = 64 real inputs (re/im of the 32 basis states),
// split into TF32 hi and lo parts.  B is the block's real 64x64 form of U
// (hi and lo), brought in by one cp.async.bulk (TMA) copy per block.  One
// thread issues 24 tcgen05.mma.kind::tf32 instructions (M=128, N=64, K=8):
// A_hi*B_hi + A_hi*B_lo + A_lo*B_hi accumulate into a 128 x 64 FP32 tile in
// tensor memory.  The readback (tcgen05.ld, one TMEM lane per tile column)
// writes every output amplitude straight into the layout the next block needs,
// or, after the last block, into natural order for the store to HBM.
// Every wait on an mbarrier is bounded; on expiry the CTA records an error,
// waits (bounded) for its own copy and MMAs, frees its tensor memory and stops.
#include <cstdio>

#include "common.hpp"
#include "tile.hpp"

namespace dq {
namespace k {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kXBytes = 32768;      // one operand copy of the tile (4096 complex64)
constexpr uint32_t kUBytes = 32768;      // U_hi + U_lo images
constexpr uint32_t kOffX0 = 0, kOffX1 = kXBytes, kOffU = 2 * kXBytes;
constexpr uint32_t kOffTabs = kOffU + kUBytes;           // lo_tab[64], hi_tab[64] (u64)
constexpr uint32_t kOffDesc = kOffTabs + 128 * 8;        // next_b[32], next_c[128] (u16)
constexpr uint32_t kOffBar = kOffDesc + 160 * 2 + 16;    // two mbarriers, 8-byte aligned
constexpr uint32_t kSmemBytes = kOffBar + 64;
constexpr uint64_t kSpinLimit = uint64_t(1) << 26;       // polls of an mbarrier before giving up
constexpr long long kWaitCycles = 4000000000LL;          // ... or this many SM cycles

struct FusedQubits {
    int q[kFusedM];
    uint16_t in_lo[64], in_hi[64];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 format, version 1):
// leading byte offset 128 (the two 16-byte K chunks of one MMA), stride byte
// offset 2048 (consecutive 8-row core-matrix groups).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr & 0x3FFFFu) >> 4);
    d |= uint64_t(128u >> 4) << 16;
    d |= uint64_t(2048u >> 4) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// kind::tf32 instruction descriptor: D FP32, A/B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false once about kWaitCycles SM cycles (about 2 s) have passed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long start = clock64();
    for (uint64_t i = 0; i < kSpinLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - start > kWaitCycles) return false;
    }
    return false;
}

__device__ __forceinline__ float tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Byte offset of complex amplitude (column, basis) in the A operand layout.
__device__ __forceinline__ uint32_t a_off(uint32_t col, uint32_t basis) {
    return (col >> 3) * 2048u + (basis >> 1) * 128u + (col & 7u) * 16u + (basis & 1u) * 8u;
}

__device__ __forceinline__ void put_split(unsigned char* sm, uint32_t off, float re, float im) {
    const float hr = tf32(re), hi = tf32(im);
    *reinterpret_cast<float2*>(sm + kOffX0 + off) = make_float2(hr, hi);
    *reinterpret_cast<float2*>(sm + kOffX1 + off) = make_float2(tf32(re - hr), tf32(im - hi));
}

__global__ void __launch_bounds__(kThreads, 2)
    k_fused(float2* __restrict__ s, int n, FusedQubits fq, const FusedBlock* __restrict__ blocks, int nblocks,
            const float* __restrict__ upool, uint64_t total_tiles, int* __restrict__ err,
            const double* __restrict__ in_norm, double* __restrict__ tile_norm) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    __shared__ double s_wsum[kThreads / 32];
    uint64_t* lo_tab = reinterpret_cast<uint64_t*>(sm + kOffTabs);
    uint64_t* hi_tab = lo_tab + 64;
    uint16_t* nb = reinterpret_cast<uint16_t*>(sm + kOffDesc);
    uint16_t* nc = nb + 32;
    const uint32_t bar_u = smem_addr(sm + kOffBar), bar_m = bar_u + 8;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int e = tid; e < 64; e += kThreads) {
        uint64_t a = 0, b = 0;
        for (int t = 0; t < 6; t++) {
            if ((e >> t) & 1) {
                a |= uint64_t(1) << fq.q[t];
                b |= uint64_t(1) << fq.q[6 + t];
            }
        }
        lo_tab[e] = a;
        hi_tab[e] = b;
    }
    if (tid == 0) {
        s_abort = 0;
        mbar_init(bar_u, 1);
        mbar_init(bar_m, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    uint32_t phase_u = 0, phase_m = 0;
    uint32_t pending_u = 0, pending_m = 0;  // issued and not yet awaited (thread 0)

    const int rest = n - kFusedM;
    for (uint64_t t = blockIdx.x; t < total_tiles && !s_abort; t += gridDim.x) {
        const uint64_t st = t >> rest;
        uint64_t tidx = t & ((uint64_t(1) << rest) - 1);
        for (int b = 0; b < kFusedM; b++) {
            uint64_t low = (uint64_t(1) << fq.q[b]) - 1;
            tidx = (tidx & low) | ((tidx & ~low) << 1);
        }
        float2* __restrict__ g = s + ((st << n) | tidx);
        // FP64 renormalisation of the previous pass (tensor-core accumulation
        // rounds toward zero, so unitary blocks shrink the norm slightly).
        const double scale = in_norm ? 1.0 / sqrt(in_norm[st]) : 1.0;
        // Tile -> A operand of block 0, split into TF32 hi / lo.
        for (uint32_t e = tid; e < 4096u; e += kThreads) {
            float2 v = g[lo_tab[e & 63] | hi_tab[e >> 6]];
            uint32_t p = uint32_t(fq.in_lo[e & 63]) | uint32_t(fq.in_hi[e >> 6]);
            put_split(sm, a_off(p >> 5, p & 31), float(double(v.x) * scale), float(double(v.y) * scale));
        }
        double norm_acc = 0.0;
        for (int j = 0; j < nblocks; j++) {
            const FusedBlock& blk = blocks[j];
            if (tid == 0) {
                // U image of this block (the previous block's MMAs are complete).
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_u), "r"(kUBytes)
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        smem_addr(sm + kOffU)),
                    "l"(upool + blk.u_off), "r"(kUBytes), "r"(bar_u)
                    : "memory");
                pending_u = 1;
            }
            if (tid < 32) nb[tid] = blk.next_b[tid];
            if (tid < 128) nc[tid] = blk.next_c[tid];
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                bool ok = mbar_wait(bar_u, phase_u & 1);
                phase_u++;
                pending_u = 0;
                if (!ok) {
                    s_abort = 1;
                    atomicExch(err, 3);
                } else {
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t ax0 = smem_addr(sm + kOffX0), ax1 = smem_addr(sm + kOffX1);
                    const uint32_t bu0 = smem_addr(sm + kOffU), bu1 = bu0 + 16384u;
#pragma unroll 1
                    for (int q = 0; q < 24; q++) {
                        const int part = q >> 3, ks = q & 7;
                        const uint32_t a = (part == 2 ? ax1 : ax0) + uint32_t(ks) * 256u;
                        const uint32_t bb = (part == 1 ? bu1 : bu0) + uint32_t(ks) * 256u;
                        const uint64_t ad = make_desc(a), bd = make_desc(bb);
                        const uint32_t acc = q > 0 ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        bar_m)
                                 : "memory");
                    pending_m = 1;
                    ok = mbar_wait(bar_m, phase_m & 1);
                    phase_m++;
                    pending_m = 0;
                    if (!ok) {
                        s_abort = 1;
                        atomicExch(err, 3);
                    }
                }
            }
            __syncthreads();
            if (s_abort) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            // Readback: warp w reads TMEM lanes 32*(w%4).. (tile columns) and
            // output columns 32*(w/4).. (16 complex outputs per thread).
            const uint32_t col = uint32_t((warp & 3) * 32 + lane);
            const uint32_t half = uint32_t(warp >> 2);
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t(warp & 3) * 32u) << 16) + half * 32u;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const uint32_t cpart = nc[col];
            if (!blk.last) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint32_t p = cpart | nb[half * 16 + i];
                    put_split(sm, a_off(p >> 5, p & 31), __uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
                }
            } else {
                float2* stage = reinterpret_cast<float2*>(sm + kOffX0);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint32_t l = cpart | nb[half * 16 + i];
                    const float re = __uint_as_float(r[2 * i]), im = __uint_as_float(r[2 * i + 1]);
                    stage[l] = make_float2(re, im);
                    norm_acc += double(re) * re + double(im) * im;
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
        }
        if (s_abort) break;
        const float2* stage = reinterpret_cast<const float2*>(sm + kOffX0);
        for (uint32_t e = tid; e < 4096u; e += kThreads) g[lo_tab[e & 63] | hi_tab[e >> 6]] = stage[e];
        // Per-tile FP64 norm, fixed-order reduction (deterministic).
        for (int o = 16; o > 0; o >>= 1) norm_acc += __shfl_down_sync(0xffffffffu, norm_acc, o);
        if (lane == 0) s_wsum[warp] = norm_acc;
        __syncthreads();
        if (tid == 0) {
            double tsum = 0.0;
            for (int w = 0; w < kThreads / 32; w++) tsum += s_wsum[w];
            tile_norm[t] = tsum;
        }
        __syncthreads();
    }
    // On an aborted wait, give the copy and the MMAs in flight a bounded chance to land.
    if (tid == 0) {
        if (pending_u) mbar_wait(bar_u, phase_u & 1);
        if (pending_m) mbar_wait(bar_m, phase_m & 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

int sm_count() {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c > 0 ? c : 148;
}

// norm[st] = sum of the state's tile norms, in tile order (one block per state).
__global__ void k_state_norm(const double* __restrict__ tile_norm, uint64_t tiles_per_state,
                             double* __restrict__ norm) {
    __shared__ double sm[256];
    const uint64_t st = blockIdx.x;
    const double* t = tile_norm + st * tiles_per_state;
    double acc = 0.0;
    for (uint64_t i = threadIdx.x; i < tiles_per_state; i += blockDim.x) acc += t[i];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) norm[st] = sm[0];
}

__global__ void k_scale_states(float2* __restrict__ s, int n, uint64_t items, const double* __restrict__ norm) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < items; g += uint64_t(gridDim.x) * blockDim.x) {
        const double sc = 1.0 / sqrt(norm[g >> n]);
        float2 v = s[g];
        s[g] = make_float2(float(double(v.x) * sc), float(double(v.y) * sc));
    }
}

}  // namespace

size_t fused_smem_bytes() { return kSmemBytes; }

void fused_state_norm(const Batch& b, const double* tile_norm, double* norm) {
    const uint64_t tiles = uint64_t(1) << (b.n - kFusedM);
    k_state_norm<<<unsigned(b.W), 256, 0, b.stream>>>(tile_norm, tiles, norm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("state norm: ") + cudaGetErrorString(e));
}

void fused_renormalize(const Batch& b, const double* norm) {
    const uint64_t items = b.W << b.n;
    const uint64_t grid = std::min<uint64_t>((items + 255) / 256, uint64_t(sm_count()) * 32);
    k_scale_states<<<unsigned(grid), 256, 0, b.stream>>>(static_cast<float2*>(b.amps), b.n, items, norm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("renormalize: ") + cudaGetErrorString(e));
}

void fused_pass(const Batch& b, const FusedPass& p, const FusedBlock* blocks_dev, const float* upool_dev, int* err,
                const double* in_norm, double* tile_norm) {
    if (!b.c64) fail(kValueError, "fused tensor-core passes run on complex64 states");
    if (b.n < kFusedM || int(p.qubits.size()) != kFusedM) fail(kValueError, "fused passes need 12 tile qubits");
    FusedQubits fq;
    for (int i = 0; i < kFusedM; i++) fq.q[i] = p.qubits[i];
    for (int e = 0; e < 64; e++) {
        fq.in_lo[e] = p.in_lo[e];
        fq.in_hi[e] = p.in_hi[e];
    }
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
        if (e != cudaSuccess) fail(kCudaError, std::string("fused pass smem: ") + cudaGetErrorString(e));
        configured = true;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused, kThreads, kSmemBytes);
    if (per_sm < 1) per_sm = 1;
    const uint64_t total = b.W << (b.n - kFusedM);
    const uint64_t grid = std::min<uint64_t>(total, uint64_t(sm_count()) * uint64_t(per_sm));
    k_fused<<<unsigned(grid), kThreads, kSmemBytes, b.stream>>>(static_cast<float2*>(b.amps), b.n, fq,
                                                               blocks_dev + p.first_block, p.nblocks, upool_dev, total,
                                                               err, in_norm, tile_norm);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("fused pass: ") + cudaGetErrorString(e));
}

}  // namespace k
}  // namespace dq

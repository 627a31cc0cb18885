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
// writes every output amplitude straight into the layout the next block needs
// (128-byte swizzled, bit orders chosen on the host to spread each half-warp's
// stores over all banks), or, after the last block, into a swizzled
// natural-order stage for the store to HBM.  The next block's gate image and
// layout tables are fetched while the current block is read back.
// Every wait on an mbarrier is bounded; on expiry the CTA records an error,
// waits (bounded) for its own copy and MMAs, frees its tensor memory and stops.
#include <algorithm>
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
constexpr uint32_t kDescBytes = 320;     // next_b[32] + next_c[128] (u16) of one block
constexpr uint32_t kOffX0 = 0, kOffX1 = kXBytes, kOffU = 2 * kXBytes;
constexpr uint32_t kOffTabs = kOffU + kUBytes;           // lo_tab[64], hi_tab[64] (u64)
constexpr uint32_t kOffIO = kOffTabs + 128 * 8;          // in_lo, in_hi, out_lo, out_hi [64] (u16)
constexpr uint32_t kOffDesc = kOffIO + 4 * 64 * 2;       // two block-table buffers
constexpr uint32_t kOffBar = kOffDesc + 2 * kDescBytes;  // two mbarriers, 8-byte aligned
constexpr uint32_t kSmemBytes = kOffBar + 64;
constexpr uint64_t kSpinLimit = uint64_t(1) << 26;       // polls of an mbarrier before giving up
constexpr long long kWaitCycles = 4000000000LL;          // ... or this many SM cycles
static_assert(kOffDesc % 16 == 0 && kDescBytes % 16 == 0, "bulk copies need 16-byte alignment");
static_assert(offsetof(FusedBlock, next_b) == 16 && sizeof(FusedBlock) % 16 == 0, "block table layout");

struct FusedQubits {
    int q[kFusedM];
    uint16_t io[4][64];  // in_lo, in_hi, out_lo, out_hi
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 format, version 1):
// leading byte offset 128 (the two 16-byte K chunks of one MMA), stride byte
// offset 2048 (consecutive 8-row core-matrix groups).  Used for the gate image.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr & 0x3FFFFu) >> 4);
    d |= uint64_t(128u >> 4) << 16;
    d |= uint64_t(2048u >> 4) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// K-major, 128-byte-swizzled descriptor (layout type 2): 8-row x 128-byte
// atoms, 1024 bytes between 8-row groups; the leading offset is unused.  The
// start address steps 32 bytes per K = 8 slice inside an atom.  Used for the tile.
__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= uint64_t((saddr & 0x3FFFFu) >> 4);
    d |= uint64_t(1) << 16;
    d |= uint64_t(1024u >> 4) << 32;
    d |= uint64_t(1) << 46;
    d |= uint64_t(2) << 61;
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

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ float tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// TF32 hi part rounded to nearest; the lo remainder is left for the tensor
// core to truncate (its error is below 2^-22 of the value).
__device__ __forceinline__ void put_split(unsigned char* sm, uint32_t off, float re, float im) {
    const float hr = tf32(re), hi = tf32(im);
    *reinterpret_cast<float2*>(sm + kOffX0 + off) = make_float2(hr, hi);
    *reinterpret_cast<float2*>(sm + kOffX1 + off) = make_float2(re - hr, im - hi);
}

// Gate image and layout tables of one block, one transaction count on bar.
__device__ __forceinline__ void fetch_block(unsigned char* sm, const FusedBlock* blk, const float* upool, uint32_t buf,
                                            uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kUBytes + kDescBytes)
                 : "memory");
    bulk_g2s(smem_addr(sm + kOffU), upool + blk->u_off, kUBytes, bar);
    bulk_g2s(smem_addr(sm + kOffDesc + buf * kDescBytes), blk->next_b, kDescBytes, bar);
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
    uint16_t* io = reinterpret_cast<uint16_t*>(sm + kOffIO);  // in_lo | in_hi | out_lo | out_hi
    const uint32_t bar_u = smem_addr(sm + kOffBar), bar_m = bar_u + 8;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid < 64) {
        uint64_t a = 0, b = 0;
        for (int t = 0; t < 6; t++) {
            if ((tid >> t) & 1) {
                a |= uint64_t(1) << fq.q[t];
                b |= uint64_t(1) << fq.q[6 + t];
            }
        }
        lo_tab[tid] = a;
        hi_tab[tid] = b;
    }
    io[tid] = fq.io[tid >> 6][tid & 63];
    if (tid == 0) {
        // The swizzled operand needs 1024-byte aligned atoms.
        s_abort = (smem_addr(sm) & 1023u) != 0;
        if (s_abort) atomicExch(err, 3);
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
    const uint64_t desc_x0 = make_desc_sw128(smem_addr(sm + kOffX0)), desc_x1 = make_desc_sw128(smem_addr(sm + kOffX1));
    const uint64_t desc_u0 = make_desc(smem_addr(sm + kOffU)), desc_u1 = make_desc(smem_addr(sm + kOffU) + 16384u);
    uint32_t phase_u = 0, phase_m = 0;
    uint32_t pending_u = 0, pending_m = 0;  // issued and not yet awaited (thread 0)
    uint32_t seq = 0;                       // blocks processed: selects the table buffer
    if (tid == 0 && uint64_t(blockIdx.x) < total_tiles) {
        fetch_block(sm, blocks, upool, 0, bar_u);
        pending_u = 1;
    }

    const int rest = n - kFusedM;
    const uint32_t row = uint32_t(tid >> 6);  // this thread's elements: l = (tid & 63) | (row + 4k) << 6
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
        const uint64_t glo = lo_tab[tid & 63];
        {
            // Tile -> A operand of block 0, split into TF32 hi / lo (loads first, all in flight).
            float2 v[16];
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = __ldcs(g + (glo | hi_tab[row + 4 * k]));
            const uint32_t plo = io[tid & 63];
#pragma unroll
            for (int k = 0; k < 16; k++)
                put_split(sm, plo ^ io[64 + row + 4 * k], float(double(v[k].x) * scale), float(double(v[k].y) * scale));
        }
        double norm_acc = 0.0;
        for (int j = 0; j < nblocks; j++) {
            const uint32_t buf = seq & 1u;
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
                    // Descriptors advance by (byte offset >> 4) in their start-address field.
#pragma unroll
                    for (int q = 0; q < 24; q++) {
                        const int part = q >> 3, ks = q & 7;
                        const uint64_t ad = (part == 2 ? desc_x1 : desc_x0) + uint64_t((ks >> 2) * 1024 + (ks & 3) * 2);
                        const uint64_t bd = (part == 1 ? desc_u1 : desc_u0) + uint64_t(ks * 16);
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                            "l"(ad), "l"(bd), "r"(kIdesc), "r"(q > 0 ? 1u : 0u));
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
                    } else {
                        // The gate image is free again: fetch the next block's while this one is read back.
                        const int next = j + 1 < nblocks ? j + 1 : (t + gridDim.x < total_tiles ? 0 : -1);
                        if (next >= 0) {
                            fetch_block(sm, blocks + next, upool, buf ^ 1u, bar_u);
                            pending_u = 1;
                        }
                    }
                }
            }
            __syncthreads();
            if (s_abort) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            // Readback: warp w reads TMEM lanes 32*(w%4).. (tile columns) and
            // output columns 32*(w/4).. (16 complex outputs per thread).
            const uint16_t* nb = reinterpret_cast<const uint16_t*>(sm + kOffDesc + buf * kDescBytes);
            const uint16_t* nc = nb + 32;
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
            uint32_t nbw[8];  // this half's 16 destination parts, two per word
            {
                const uint4 w0 = *reinterpret_cast<const uint4*>(nb + half * 16);
                const uint4 w1 = *reinterpret_cast<const uint4*>(nb + half * 16 + 8);
                nbw[0] = w0.x, nbw[1] = w0.y, nbw[2] = w0.z, nbw[3] = w0.w;
                nbw[4] = w1.x, nbw[5] = w1.y, nbw[6] = w1.z, nbw[7] = w1.w;
            }
            if (j + 1 < nblocks) {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint32_t off = cpart ^ ((nbw[i >> 1] >> (16 * (i & 1))) & 0xFFFFu);
                    put_split(sm, off, __uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
                }
            } else {
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const uint32_t off = cpart ^ ((nbw[i >> 1] >> (16 * (i & 1))) & 0xFFFFu);
                    const float re = __uint_as_float(r[2 * i]), im = __uint_as_float(r[2 * i + 1]);
                    *reinterpret_cast<float2*>(sm + kOffX0 + off) = make_float2(re, im);
                    norm_acc += double(re) * re + double(im) * im;
                }
            }
            seq++;
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncthreads();
        }
        if (s_abort) break;
        const uint32_t olo = io[128 + (tid & 63)];
#pragma unroll
        for (int k = 0; k < 16; k++)
            g[glo | hi_tab[row + 4 * k]] = *reinterpret_cast<const float2*>(sm + kOffX0 + (olo ^ io[192 + row + 4 * k]));
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
    // On an aborted wait, give the copies and the MMAs in flight a bounded chance to land.
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
        fq.io[0][e] = p.in_lo[e];
        fq.io[1][e] = p.in_hi[e];
        fq.io[2][e] = p.out_lo[e];
        fq.io[3][e] = p.out_hi[e];
    }
    // Two CTAs per SM need the largest shared-memory carveout.  Residency is
    // computed from the kernel's registers and shared memory (the grid-stride
    // loop is correct for any grid; a grid below residency leaves SMs half idle).
    static int per_sm_of[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& per_sm = per_sm_of[dev & 63];
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_fused, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     int(cudaSharedmemCarveoutMaxShared));
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_fused);
        int smem_sm = 0, reserved = 0, regs_sm = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        if (e != cudaSuccess) fail(kCudaError, std::string("fused pass setup: ") + cudaGetErrorString(e));
        const size_t per_cta = kSmemBytes + fa.sharedSizeBytes + size_t(reserved);
        const int by_smem = int(size_t(smem_sm) / per_cta);
        const int by_regs = fa.numRegs > 0 ? regs_sm / (fa.numRegs * kThreads) : 2;
        per_sm = std::max(1, std::min({2, by_smem, by_regs}));
    }
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

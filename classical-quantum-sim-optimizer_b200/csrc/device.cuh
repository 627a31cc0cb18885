// Device-side helpers: complex arithmetic on interleaved amplitudes, index
// expansion, classical-condition evaluation and the ChaCha8 stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dq {
namespace dev {

// ---- complex arithmetic (interleaved re/im, 16 B for c128, 8 B for c64) ----
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, double s) {
    return make_float2(float(double(a.x) * s), float(double(a.y) * s));
}
__device__ __forceinline__ double norm2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double norm2(float2 a) {
    double x = a.x, y = a.y;
    return x * x + y * y;
}
template <typename V> __device__ __forceinline__ V czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }
template <typename V> __device__ __forceinline__ V from_d2(double2 a);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 a) { return make_float2(float(a.x), float(a.y)); }

// ---- index helpers ----
// Ascending bit positions at which a compact index gets zero bits inserted
// (the reference's insert_target_zeros, src/engine.rs:245-251).
struct InsertSet {
    int k;
    int pos[8];
};

__device__ __forceinline__ uint64_t expand(uint64_t j, const InsertSet& s) {
#pragma unroll
    for (int t = 0; t < 8; t++) {
        if (t < s.k) {
            uint64_t low = (uint64_t(1) << s.pos[t]) - 1;
            j = (j & low) | ((j & ~low) << 1);
        }
    }
    return j;
}

// ---- classical conditions (nested conditionals are an AND of entries) ----
struct CondList {
    int n;
    uint32_t size[6];
    uint64_t base[6];
    uint64_t value[6];
};

__device__ __forceinline__ uint64_t extract_bits(const uint64_t* w, uint64_t base, uint32_t size) {
    uint64_t wi = base >> 6;
    uint32_t off = uint32_t(base & 63);
    uint64_t v = w[wi] >> off;
    if (off != 0 && off + size > 64) v |= w[wi + 1] << (64 - off);
    return size >= 64 ? v : (v & ((uint64_t(1) << size) - 1));
}

// True when every condition holds for state `st` (cbits packed LSB-first, cwords per state).
__device__ __forceinline__ bool cond_ok(const CondList& c, const uint64_t* cbits, int cwords, uint64_t st) {
    const uint64_t* w = cbits + st * uint64_t(cwords);
    // Constant indices keep the table in parameter space (no local-memory copy).
#pragma unroll
    for (int t = 0; t < 6; t++) {
        if (t >= c.n) break;
        if (extract_bits(w, c.base[t], c.size[t]) != c.value[t]) return false;
    }
    return true;
}

// ---- ChaCha8 (rand_chacha 0.3 layout) seeded by rand_core's seed_from_u64 ----
__device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

#define DQ_QR(a, b, c, d) \
    a += b;               \
    d ^= a;               \
    d = rotl32(d, 16);    \
    c += d;               \
    b ^= c;               \
    b = rotl32(b, 12);    \
    a += b;               \
    d ^= a;               \
    d = rotl32(d, 8);     \
    c += d;               \
    b ^= c;               \
    b = rotl32(b, 7);

// Two consecutive words (2*kk, 2*kk+1) of the ChaCha8 stream keyed by
// seed_from_u64(seed), combined as next_u64 does: low word first.
__device__ __forceinline__ uint64_t chacha8_u64(uint64_t seed, uint64_t kk) {
    uint32_t key[8];
    uint64_t st = seed;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        st = st * 6364136223846793005ULL + 11634580027462260723ULL;
        uint32_t xs = uint32_t(((st >> 18) ^ st) >> 27);
        uint32_t rot = uint32_t(st >> 59);
        key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
    }
    uint64_t w = 2 * kk;
    uint64_t block = w >> 4;
    uint32_t in[16];
    in[0] = 0x61707865u;
    in[1] = 0x3320646eu;
    in[2] = 0x79622d32u;
    in[3] = 0x6b206574u;
#pragma unroll
    for (int i = 0; i < 8; i++) in[4 + i] = key[i];
    in[12] = uint32_t(block);
    in[13] = uint32_t(block >> 32);
    in[14] = 0;
    in[15] = 0;
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = in[i];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        DQ_QR(x[0], x[4], x[8], x[12]);
        DQ_QR(x[1], x[5], x[9], x[13]);
        DQ_QR(x[2], x[6], x[10], x[14]);
        DQ_QR(x[3], x[7], x[11], x[15]);
        DQ_QR(x[0], x[5], x[10], x[15]);
        DQ_QR(x[1], x[6], x[11], x[12]);
        DQ_QR(x[2], x[7], x[8], x[13]);
        DQ_QR(x[3], x[4], x[9], x[14]);
    }
    uint32_t sel = uint32_t(w & 15);  // even: words sel and sel+1 of this block
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
        if (uint32_t(i) == sel) {
            lo = x[i] + in[i];
            hi = x[i + 1] + in[i + 1];
        }
    }
    return (uint64_t(hi) << 32) | lo;
}
#undef DQ_QR

// rand 0.8 Standard f64: 53 high bits scaled by 2^-53.
__device__ __forceinline__ double u64_to_unit(uint64_t v) { return double(v >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace dev
}  // namespace dq

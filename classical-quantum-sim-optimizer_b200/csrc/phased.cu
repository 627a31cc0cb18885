// Tile passes in register phases: host grouping and the sm_100a kernel.
#include "phased.hpp"

#include <algorithm>
#include <cstring>
#include <string>

#include "common.hpp"

namespace dq {

namespace {

int popcount32(uint32_t x) { return __builtin_popcount(x); }

// Tile bits whose amplitudes an operation mixes (T) and every bit it reads (S).
void op_masks(const TileOp& t, uint32_t& T, uint32_t& S) {
    S = 0;
    for (int i = 0; i < t.nins; i++) S |= 1u << t.ins[i];
    switch (t.type) {
        case TileOp::kOne:
        case TileOp::kX: T = t.tbit; break;
        case TileOp::kSwap: T = t.lowbit | t.highbit; break;
        case TileOp::kDense:
            T = 0;
            for (int b = 0; b < t.k; b++) T |= 1u << t.q[b];
            S |= T;
            break;
        case TileOp::kDiagFull:
            T = 0;
            for (int b = 0; b < t.k; b++) S |= 1u << t.q[b];
            break;
        default: T = 0; break;  // kDiagEntry: a pattern on its ins bits
    }
}

// Register index of tile bit `bit` among the phase's register qubits R (ascending).
int reg_of(const int R[kPhaseRegBits], int bit) {
    for (int i = 0; i < kPhaseRegBits; i++)
        if (R[i] == bit) return i;
    fail(kValueError, "phase operation outside its register qubits");
    return -1;
}

// Dense matrix of 2 or 3 qubits re-laid out so that matrix index bit j sits on
// the op's j-th lowest register qubit; sets the phase code.
std::vector<double2> canonical_dense(const TileOp& t, const int R[kPhaseRegBits], const std::vector<double2>& pool,
                                     int& code) {
    const int k = t.k, D = 1 << k;
    int reg[3] = {0, 0, 0};  // register index of matrix bit (k-1-b) = op qubit q[b]
    for (int b = 0; b < k; b++) reg[b] = reg_of(R, t.q[b]);
    int sorted[3] = {reg[0], reg[1], reg[2]};
    std::sort(sorted, sorted + k);
    // Original matrix index of canonical index x.
    auto orig = [&](int x) {
        int y = 0;
        for (int b = 0; b < k; b++) {
            const int j = int(std::find(sorted, sorted + k, reg[b]) - sorted);  // canonical bit of q[b]
            if ((x >> j) & 1) y |= 1 << (k - 1 - b);
        }
        return y;
    };
    code = k == 2 ? kPhD2 + phase_pair(sorted[1], sorted[0]) : kPhD3 + phase_triple(sorted[2], sorted[1], sorted[0]);
    std::vector<double2> out;
    for (int x = 0; x < D; x++)
        for (int xc = 0; xc < D; xc++) out.push_back(pool[size_t(t.mat) + size_t(orig(x)) * D + orig(xc)]);
    return out;
}

struct PendingOp {
    int code = 0, k = 0;
    uint32_t mask = 0, value = 0;
    uint8_t q[8] = {};
    std::vector<double2> mat;
};

struct PendingPhase {
    int R[kPhaseRegBits] = {};
    std::vector<int> ord;  // slot bit i -> tile bit
    std::vector<PendingOp> ops;
};

uint4 word(uint32_t x, uint32_t y, uint32_t z, uint32_t w) { return make_uint4(x, y, z, w); }

}  // namespace

int plan_phases(const std::vector<TileOp>& ops, int m, bool c64, const std::vector<double2>& pool,
                std::vector<uint4>& block) {
    const int N = int(ops.size());
    const int g = c64 ? 4 : 3;
    std::vector<uint32_t> T(N), S(N);
    for (int i = 0; i < N; i++) op_masks(ops[i], T[i], S[i]);
    std::vector<char> done(N, 0);
    int left = N;
    // Operations a phase with register qubits R takes: one scan in pass order;
    // an operation joins when its targets lie in R and it commutes with every
    // operation skipped before it, and a skipped operation blocks what
    // depends on it.
    std::vector<int> members, best;
    auto scan = [&](uint32_t R, std::vector<int>& out) {
        out.clear();
        uint32_t blockT = 0, blockS = 0;
        for (int i = 0; i < N; i++) {
            if (done[i]) continue;
            if ((T[i] & ~R) == 0 && !(T[i] & blockS) && !(S[i] & blockT)) {
                out.push_back(i);
            } else {
                blockT |= T[i];
                blockS |= S[i];
            }
        }
    };
    const uint32_t all = m >= 32 ? ~0u : (1u << m) - 1;
    std::vector<PendingPhase> phases;
    while (left > 0) {
        // Candidate register sets: the targets of each operation that is ready
        // (commutes with every earlier one left), widened to kPhaseRegBits
        // qubits in every way.  The set whose phase takes the most operations
        // wins.
        std::vector<uint32_t> ready;
        {
            uint32_t blockT = 0, blockS = 0;
            for (int i = 0; i < N; i++) {
                if (done[i]) continue;
                if (!(T[i] & blockS) && !(S[i] & blockT)) ready.push_back(T[i]);
                blockT |= T[i];
                blockS |= S[i];
            }
        }
        std::vector<uint32_t> cands;
        auto widen = [&](uint32_t R, auto&& self) -> void {
            if (popcount32(R) >= kPhaseRegBits) {
                cands.push_back(R);
                return;
            }
            for (int b = 0; b < m; b++)
                if (((all >> b) & 1) && !((R >> b) & 1)) self(R | (1u << b), self);
        };
        for (uint32_t x : ready)
            if (x && popcount32(x) <= kPhaseRegBits) widen(x, widen);
        std::sort(cands.begin(), cands.end());
        cands.erase(std::unique(cands.begin(), cands.end()), cands.end());
        if (cands.empty()) cands.push_back(0);  // only diagonal operations are ready
        best.clear();
        uint32_t R = 0;
        for (uint32_t c : cands) {
            scan(c, members);
            if (members.size() > best.size()) {
                best.swap(members);
                R = c;
            }
        }
        members.swap(best);
        // Pad the register qubits with unused tile bits, highest first.
        for (int b = m - 1; b >= 0 && popcount32(R) < kPhaseRegBits; b--)
            if (!((R >> b) & 1)) R |= 1u << b;
        PendingPhase ph;
        for (int b = 0, nr = 0; b < m; b++)
            if ((R >> b) & 1) ph.R[nr++] = b;
        // Slot bits: first one tile bit of each residue mod g (lowest first), so
        // the 2^g lanes of a shared-memory wavefront hit distinct bank groups;
        // then the other free bits ascending.
        std::vector<char> used(size_t(m), 0);
        for (int cls = 0; cls < g; cls++)
            for (int b = cls; b < m; b += g)
                if (!((R >> b) & 1)) {
                    ph.ord.push_back(b);
                    used[size_t(b)] = 1;
                    break;
                }
        for (int b = 0; b < m; b++)
            if (!((R >> b) & 1) && !used[size_t(b)]) ph.ord.push_back(b);
        for (int i : members) {
            const TileOp& t = ops[size_t(i)];
            PendingOp p;
            auto copy_mat = [&](int count) {
                for (int e = 0; e < count; e++) p.mat.push_back(pool[size_t(t.mat) + size_t(e)]);
            };
            switch (t.type) {
                case TileOp::kOne:
                case TileOp::kX:
                    p.code = (t.type == TileOp::kOne ? kPhOne : kPhX) + reg_of(ph.R, __builtin_ctz(t.tbit));
                    if (t.type == TileOp::kOne) copy_mat(4);
                    p.mask = S[size_t(i)] & ~t.tbit;
                    p.value = t.fixed;
                    break;
                case TileOp::kSwap:
                    p.code = kPhSwap + phase_pair(reg_of(ph.R, __builtin_ctz(t.highbit)),
                                                  reg_of(ph.R, __builtin_ctz(t.lowbit)));
                    p.mask = S[size_t(i)] & ~(t.lowbit | t.highbit);
                    p.value = t.fixed;
                    break;
                case TileOp::kDiagEntry:
                    p.code = kPhDiagEntry;
                    copy_mat(1);
                    p.mask = S[size_t(i)];
                    p.value = t.fixed;
                    break;
                case TileOp::kDiagFull:
                    p.code = kPhDiagFull;
                    p.k = t.k;
                    for (int b = 0; b < t.k; b++) p.q[b] = uint8_t(t.q[b]);
                    copy_mat(1 << t.k);
                    break;
                case TileOp::kDense:
                    if (t.k == 1) {
                        p.code = kPhOne + reg_of(ph.R, t.q[0]);
                        copy_mat(4);  // row-major 2x2: u00, u01, u10, u11
                    } else {
                        p.mat = canonical_dense(t, ph.R, pool, p.code);
                    }
                    break;
                default: fail(kValueError, "tile operation without a phase form");
            }
            ph.ops.push_back(std::move(p));
            done[size_t(i)] = 1;
        }
        left -= int(members.size());
        phases.push_back(std::move(ph));
    }
    // Assemble the block: phase headers, then operations, then matrices.
    const size_t nph = phases.size();
    size_t op_word = nph * kPhaseWords;
    block.assign(op_word + size_t(N) * kPhaseOpWords, make_uint4(0, 0, 0, 0));
    for (size_t pi = 0; pi < nph; pi++) {
        const PendingPhase& ph = phases[pi];
        uint4* h = &block[pi * kPhaseWords];
        h[0] = word(uint32_t(op_word), uint32_t(ph.ops.size()), uint32_t(ph.ord.size()), 0);
        uint32_t rp[4] = {0, 0, 0, 0}, sp[kPhaseMaxSlotBits] = {};
        for (int i = 0; i < kPhaseRegBits; i++) rp[i] = (1u << ph.R[i]) | (phase_swizzle(1u << ph.R[i], g) << 16);
        for (size_t i = 0; i < ph.ord.size(); i++)
            sp[i] = (1u << ph.ord[i]) | (phase_swizzle(1u << ph.ord[i], g) << 16);
        h[1] = word(rp[0], rp[1], rp[2], rp[3]);
        for (int q4 = 0; q4 < 4; q4++) h[2 + q4] = word(sp[4 * q4], sp[4 * q4 + 1], sp[4 * q4 + 2], sp[4 * q4 + 3]);
        for (const PendingOp& p : ph.ops) {
            uint32_t q0 = 0, q1 = 0;
            for (int b = 0; b < 4; b++) {
                q0 |= uint32_t(p.q[b]) << (8 * b);
                q1 |= uint32_t(p.q[4 + b]) << (8 * b);
            }
            block[op_word] = word(uint32_t(p.code), p.mat.empty() ? 0u : uint32_t(block.size()), p.mask, p.value);
            block[op_word + 1] = word(uint32_t(p.k), q0, q1, 0);
            op_word += kPhaseOpWords;
            for (const double2& v : p.mat) {
                uint4 u;
                std::memcpy(&u, &v, sizeof u);
                block.push_back(u);
            }
        }
    }
    return int(nph);
}

namespace k {
namespace {

constexpr int kPhaseThreads = 256;
constexpr int E = kPhaseEntries;

struct PhaseQubits {
    int m;
    int q[20];
};

// The block as a launch argument (constant bank).
struct PhasedArgs {
    uint4 q[kPhaseParamWords];
};

// Word sources: the block in device memory, or the launch argument.
struct DevWords {
    const uint4* __restrict__ w;
    __device__ __forceinline__ uint4 operator()(int i) const { return __ldg(w + i); }
};
struct ArgWords {
    const PhasedArgs* a;
    __device__ __forceinline__ uint4 operator()(int i) const { return a->q[i]; }
};

template <typename V>
__device__ __forceinline__ V mat_of(uint4 u) {
    return dev::from_d2<V>(make_double2(__hiloint2double(int(u.y), int(u.x)), __hiloint2double(int(u.w), int(u.z))));
}

// acc += m * v as four fused multiply-adds (the products are not rounded
// before the sum).
__device__ __forceinline__ void cmac(double2& acc, double2 m, double2 v) {
    acc.x = fma(m.x, v.x, acc.x);
    acc.x = fma(-m.y, v.y, acc.x);
    acc.y = fma(m.x, v.y, acc.y);
    acc.y = fma(m.y, v.x, acc.y);
}
__device__ __forceinline__ void cmac(float2& acc, float2 m, float2 v) {
    acc.x = fmaf(m.x, v.x, acc.x);
    acc.x = fmaf(-m.y, v.y, acc.x);
    acc.y = fmaf(m.x, v.y, acc.y);
    acc.y = fmaf(m.y, v.x, acc.y);
}

// One operation of a phase: its first matrix word and its condition.
struct Op {
    int code, mat;
    uint32_t mask, value;
};

template <typename V, int T, class W>
__device__ __forceinline__ void ph_one(V (&a)[E], const W& w, const Op& op, uint32_t base, const uint32_t (&rb)[E]) {
    const V u00 = mat_of<V>(w(op.mat)), u01 = mat_of<V>(w(op.mat + 1));
    const V u10 = mat_of<V>(w(op.mat + 2)), u11 = mat_of<V>(w(op.mat + 3));
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & (1 << T)) continue;
        const int u = v | (1 << T);
        if (op.mask && ((base | rb[v]) & op.mask) != op.value) continue;
        const V x = a[v], y = a[u];
        V p = dev::czero<V>(), q = dev::czero<V>();
        cmac(p, u00, x);
        cmac(p, u01, y);
        cmac(q, u10, x);
        cmac(q, u11, y);
        a[v] = p;
        a[u] = q;
    }
}

template <typename V, int T>
__device__ __forceinline__ void ph_x(V (&a)[E], const Op& op, uint32_t base, const uint32_t (&rb)[E]) {
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & (1 << T)) continue;
        const int u = v | (1 << T);
        if (op.mask && ((base | rb[v]) & op.mask) != op.value) continue;
        const V x = a[v];
        a[v] = a[u];
        a[u] = x;
    }
}

template <typename V, int H, int L>
__device__ __forceinline__ void ph_swap(V (&a)[E], const Op& op, uint32_t base, const uint32_t (&rb)[E]) {
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & ((1 << H) | (1 << L))) continue;
        const int v01 = v | (1 << L), v10 = v | (1 << H);
        if (op.mask && ((base | rb[v01]) & op.mask) != op.value) continue;
        const V x = a[v01];
        a[v01] = a[v10];
        a[v10] = x;
    }
}

// Dense matrix of K = 2 or 3 qubits on register qubits Q0 > Q1 (> Q2)
// (matrix index bit K-1-b on the b-th), applied to every group of the other
// register qubits.  Rows are read one at a time; all groups' outputs are
// formed before any is written back.
template <typename V, int K, int Q0, int Q1, int Q2, class W>
__device__ __forceinline__ void ph_dense(V (&a)[E], const W& w, const Op& op) {
    constexpr int D = 1 << K;
    constexpr int QM = (1 << Q0) | (1 << Q1) | (K == 3 ? (1 << Q2) : 0);
    constexpr int G = E / D;
    auto entry = [](int g0, int c) {
        return K == 3 ? (g0 | (((c >> 2) & 1) << Q0) | (((c >> 1) & 1) << Q1) | ((c & 1) << Q2))
                      : (g0 | (((c >> 1) & 1) << Q0) | ((c & 1) << Q1));
    };
    int gbase[G];
    {
        int gi = 0;
#pragma unroll
        for (int v = 0; v < E; v++)
            if (!(v & QM)) gbase[gi++] = v;
    }
    V out[E];
#pragma unroll
    for (int r = 0; r < D; r++) {
        V mr[D];
#pragma unroll
        for (int c = 0; c < D; c++) mr[c] = mat_of<V>(w(op.mat + r * D + c));
#pragma unroll
        for (int gi = 0; gi < G; gi++) {
            V acc = dev::czero<V>();
#pragma unroll
            for (int c = 0; c < D; c++) cmac(acc, mr[c], a[entry(gbase[gi], c)]);
            out[entry(gbase[gi], r)] = acc;
        }
    }
#pragma unroll
    for (int v = 0; v < E; v++) a[v] = out[v];
}

template <typename V, class W>
__device__ __forceinline__ void ph_diag_entry(V (&a)[E], const W& w, const Op& op, uint32_t base,
                                              const uint32_t (&rb)[E]) {
    const V d = mat_of<V>(w(op.mat));
#pragma unroll
    for (int v = 0; v < E; v++)
        if (((base | rb[v]) & op.mask) == op.value) a[v] = dev::cmul(a[v], d);
}

// A full diagonal: `extra` = {k, table qubits 0-3 and 4-7 as bytes}.
template <typename V, class W>
__device__ __forceinline__ void ph_diag_full(V (&a)[E], const W& w, const Op& op, uint4 extra, uint32_t base,
                                             const uint32_t (&rb)[E]) {
    const int k = int(extra.x);
#pragma unroll
    for (int v = 0; v < E; v++) {
        const uint32_t full = base | rb[v];
        uint32_t jj = 0;
#pragma unroll
        for (int b = 0; b < 8; b++)
            if (b < k) jj = (jj << 1) | ((full >> (((b < 4 ? extra.y : extra.z) >> (8 * (b & 3))) & 0xFFu)) & 1u);
        a[v] = dev::cmul(a[v], mat_of<V>(w(op.mat + int(jj))));
    }
}

template <typename V, class W>
__device__ __forceinline__ void ph_apply(V (&a)[E], const W& w, int opw, uint32_t base, const uint32_t (&rb)[E]) {
    const uint4 h = w(opw);
    const Op op{int(h.x), int(h.y), h.z, h.w};
    switch (op.code) {
        case kPhOne + 0: ph_one<V, 0>(a, w, op, base, rb); break;
        case kPhOne + 1: ph_one<V, 1>(a, w, op, base, rb); break;
        case kPhOne + 2: ph_one<V, 2>(a, w, op, base, rb); break;
        case kPhX + 0: ph_x<V, 0>(a, op, base, rb); break;
        case kPhX + 1: ph_x<V, 1>(a, op, base, rb); break;
        case kPhX + 2: ph_x<V, 2>(a, op, base, rb); break;
        case kPhD2 + phase_pair(1, 0): ph_dense<V, 2, 1, 0, 0>(a, w, op); break;
        case kPhD2 + phase_pair(2, 0): ph_dense<V, 2, 2, 0, 0>(a, w, op); break;
        case kPhD2 + phase_pair(2, 1): ph_dense<V, 2, 2, 1, 0>(a, w, op); break;
        case kPhD3 + phase_triple(2, 1, 0): ph_dense<V, 3, 2, 1, 0>(a, w, op); break;
        case kPhSwap + phase_pair(1, 0): ph_swap<V, 1, 0>(a, op, base, rb); break;
        case kPhSwap + phase_pair(2, 0): ph_swap<V, 2, 0>(a, op, base, rb); break;
        case kPhSwap + phase_pair(2, 1): ph_swap<V, 2, 1>(a, op, base, rb); break;
#if DQ_PHASE_REG_BITS == 4
        case kPhOne + 3: ph_one<V, 3>(a, w, op, base, rb); break;
        case kPhX + 3: ph_x<V, 3>(a, op, base, rb); break;
        case kPhD2 + phase_pair(3, 0): ph_dense<V, 2, 3, 0, 0>(a, w, op); break;
        case kPhD2 + phase_pair(3, 1): ph_dense<V, 2, 3, 1, 0>(a, w, op); break;
        case kPhD2 + phase_pair(3, 2): ph_dense<V, 2, 3, 2, 0>(a, w, op); break;
        case kPhD3 + phase_triple(3, 1, 0): ph_dense<V, 3, 3, 1, 0>(a, w, op); break;
        case kPhD3 + phase_triple(3, 2, 0): ph_dense<V, 3, 3, 2, 0>(a, w, op); break;
        case kPhD3 + phase_triple(3, 2, 1): ph_dense<V, 3, 3, 2, 1>(a, w, op); break;
        case kPhSwap + phase_pair(3, 0): ph_swap<V, 3, 0>(a, op, base, rb); break;
        case kPhSwap + phase_pair(3, 1): ph_swap<V, 3, 1>(a, op, base, rb); break;
        case kPhSwap + phase_pair(3, 2): ph_swap<V, 3, 2>(a, op, base, rb); break;
#endif
        case kPhDiagEntry: ph_diag_entry<V>(a, w, op, base, rb); break;
        case kPhDiagFull: ph_diag_full<V>(a, w, op, w(opw + 1), base, rb); break;
        default: break;
    }
}

template <typename V>
__device__ __forceinline__ uint32_t swz(uint32_t e) {
    constexpr int g = sizeof(V) == 16 ? 3 : 4;
    uint32_t f = 0;
#pragma unroll
    for (int s = g; s < 20; s += g) f ^= e >> s;
    return e ^ (f & ((1u << g) - 1));
}

// The persistent pass: each CTA loads a tile into (swizzled) shared memory,
// runs the phases and writes the tile back.
template <typename V, class W>
__device__ __forceinline__ void phased_body(V* __restrict__ s, int n, int m, const PhaseQubits& tq, int nphases,
                                            uint64_t total_tiles, const W& w) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    const int lb = m < 6 ? m : 6;
    uint64_t* lo_tab = reinterpret_cast<uint64_t*>(smem_raw + (sizeof(V) << m));
    uint64_t* hi_tab = lo_tab + (1 << lb);
    for (int e = threadIdx.x; e < (1 << lb); e += blockDim.x) {
        uint64_t off = 0;
        for (int b = 0; b < lb; b++)
            if ((e >> b) & 1) off |= uint64_t(1) << tq.q[b];
        lo_tab[e] = off;
    }
    for (int e = threadIdx.x; e < (1 << (m - lb)); e += blockDim.x) {
        uint64_t off = 0;
        for (int b = 0; b < m - lb; b++)
            if ((e >> b) & 1) off |= uint64_t(1) << tq.q[lb + b];
        hi_tab[e] = off;
    }
    __syncthreads();
    const int rest = n - m;
    const uint32_t size = 1u << m, slots = size >> kPhaseRegBits;
    const uint32_t lmask = (1u << lb) - 1;
    for (uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint64_t st = t >> rest;
        uint64_t tid = t & ((uint64_t(1) << rest) - 1);
        for (int b = 0; b < m; b++) {
            uint64_t low = (uint64_t(1) << tq.q[b]) - 1;
            tid = (tid & low) | ((tid & ~low) << 1);
        }
        V* __restrict__ gp = s + ((st << n) | tid);
        constexpr int U = 4;
        for (uint32_t e0 = threadIdx.x; e0 < size; e0 += blockDim.x * U) {
            V r[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t e = e0 + u * blockDim.x;
                if (e < size) r[u] = gp[lo_tab[e & lmask] | hi_tab[e >> lb]];
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const uint32_t e = e0 + u * blockDim.x;
                if (e < size) tile[swz<V>(e)] = r[u];
            }
        }
        __syncthreads();
        for (int p = 0; p < nphases; p++) {
            const uint4 h0 = w(kPhaseWords * p), h1 = w(kPhaseWords * p + 1);
            const int first = int(h0.x), nops = int(h0.y), nsb = int(h0.z);
            const uint32_t rp[4] = {h1.x, h1.y, h1.z, h1.w};
            // Register entry v: tile offset and swizzled offset (ORs / XORs of
            // its register qubits' bits).
            uint32_t rb[E], prb[E];
#pragma unroll
            for (int v = 0; v < E; v++) {
                uint32_t o = 0, po = 0;
#pragma unroll
                for (int i = 0; i < kPhaseRegBits; i++)
                    if ((v >> i) & 1) {
                        o |= rp[i] & 0xFFFFu;
                        po ^= rp[i] >> 16;
                    }
                rb[v] = o;
                prb[v] = po;
            }
            for (uint32_t sl = threadIdx.x; sl < slots; sl += blockDim.x) {
                uint32_t base = 0, pbase = 0;
#pragma unroll
                for (int q4 = 0; q4 < kPhaseMaxSlotBits / 4; q4++) {
                    if (4 * q4 >= nsb) break;
                    const uint4 sw = w(kPhaseWords * p + 2 + q4);
                    const uint32_t spk[4] = {sw.x, sw.y, sw.z, sw.w};
#pragma unroll
                    for (int j = 0; j < 4; j++)
                        if (4 * q4 + j < nsb && ((sl >> (4 * q4 + j)) & 1u)) {
                            base |= spk[j] & 0xFFFFu;
                            pbase ^= spk[j] >> 16;
                        }
                }
                V a[E];
#pragma unroll
                for (int v = 0; v < E; v++) a[v] = tile[pbase ^ prb[v]];
                for (int o = 0; o < nops; o++) ph_apply<V>(a, w, first + kPhaseOpWords * o, base, rb);
#pragma unroll
                for (int v = 0; v < E; v++) tile[pbase ^ prb[v]] = a[v];
            }
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) gp[lo_tab[e & lmask] | hi_tab[e >> lb]] = tile[swz<V>(e)];
        __syncthreads();
    }
}

// Resident CTAs per SM the register allocation is bounded for: complex128 tiles
// (64 KB of shared memory each at 12 tile qubits) take DQ_PHASE_CTAS_C128.
#ifndef DQ_PHASE_CTAS_C128
#define DQ_PHASE_CTAS_C128 2
#endif
template <typename V>
constexpr int phase_min_ctas() {
    return sizeof(V) == 16 ? (kPhaseRegBits == 3 ? DQ_PHASE_CTAS_C128 : 1) : 2;
}

template <typename V>
__global__ void __launch_bounds__(kPhaseThreads, phase_min_ctas<V>())
    k_tile_phased_dev(V* __restrict__ s, int n, int m, PhaseQubits tq, int nphases, uint64_t total_tiles,
                      const uint4* __restrict__ block) {
    phased_body<V>(s, n, m, tq, nphases, total_tiles, DevWords{block});
}

template <typename V>
__global__ void __launch_bounds__(kPhaseThreads, phase_min_ctas<V>())
    k_tile_phased_arg(V* __restrict__ s, int n, int m, PhaseQubits tq, int nphases, uint64_t total_tiles,
                      const __grid_constant__ PhasedArgs args) {
    phased_body<V>(s, n, m, tq, nphases, total_tiles, ArgWords{&args});
}

int sm_count() {
    static int c = 0;
    if (!c) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
        if (c <= 0) c = 148;
    }
    return c;
}

template <typename Kernel>
uint64_t configure(Kernel kernel, size_t smem, size_t& configured, uint64_t total) {
    if (smem > configured) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
        configured = smem;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPhaseThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return std::min<uint64_t>(total, uint64_t(sm_count()) * per_sm);
}

template <typename V>
void launch_phased(const Batch& b, const TilePass& hp, int nphases, const std::vector<uint4>& block,
                   const uint4* block_dev) {
    const int m = int(hp.qubits.size());
    if (!phase_supported(m)) fail(kValueError, "tile pass too small or too large for register phases");
    PhaseQubits tq{};
    tq.m = m;
    for (int i = 0; i < m; i++) tq.q[i] = hp.qubits[size_t(i)];
    const size_t smem = tile_smem_bytes(m, sizeof(V) == 8);
    const uint64_t total = b.W << (b.n - m);
    if (block.size() <= size_t(kPhaseParamWords)) {
        static size_t configured = 0;
        const uint64_t grid = configure(k_tile_phased_arg<V>, smem, configured, total);
        static thread_local PhasedArgs args;
        std::memcpy(args.q, block.data(), block.size() * sizeof(uint4));
        k_tile_phased_arg<V><<<unsigned(grid), kPhaseThreads, smem, b.stream>>>(static_cast<V*>(b.amps), b.n, m, tq,
                                                                                 nphases, total, args);
    } else {
        if (!block_dev) fail(kValueError, "phased tile pass without its device block");
        static size_t configured = 0;
        const uint64_t grid = configure(k_tile_phased_dev<V>, smem, configured, total);
        k_tile_phased_dev<V><<<unsigned(grid), kPhaseThreads, smem, b.stream>>>(static_cast<V*>(b.amps), b.n, m, tq,
                                                                                 nphases, total, block_dev);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("phased tile pass: ") + cudaGetErrorString(e));
}

}  // namespace

void tile_pass_phased(const Batch& b, const TilePass& host_pass, int nphases, const std::vector<uint4>& block,
                      const uint4* block_dev) {
    if (b.c64)
        launch_phased<float2>(b, host_pass, nphases, block, block_dev);
    else
        launch_phased<double2>(b, host_pass, nphases, block, block_dev);
}

}  // namespace k
}  // namespace dq

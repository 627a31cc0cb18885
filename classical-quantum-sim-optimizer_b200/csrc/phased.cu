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

// Register index (0..3) of tile bit `bit` among the phase's register qubits R (ascending).
int reg_of(const int R[kPhaseRegBits], int bit) {
    for (int i = 0; i < kPhaseRegBits; i++)
        if (R[i] == bit) return i;
    fail(kValueError, "phase operation outside its register qubits");
    return -1;
}

// Dense matrix of 2 or 3 qubits re-laid out so that matrix index bit j sits on
// the op's j-th lowest register qubit; sets the phase code, returns the pool
// offset.
int canonical_dense(const TileOp& t, const int R[kPhaseRegBits], const std::vector<double2>& src_pool,
                    std::vector<double2>& pool, int& code) {
    const int k = t.k, D = 1 << k;
    int reg[3] = {0, 0, 0};  // register index of matrix bit (k-1-b) = op qubit q[b]
    for (int b = 0; b < k; b++) reg[b] = reg_of(R, t.q[b]);
    // Canonical order: matrix bit j <-> the j-th smallest register index of the op.
    int sorted[3] = {reg[0], reg[1], reg[2]};
    std::sort(sorted, sorted + k);
    // y(x): original matrix index of canonical index x.
    auto orig = [&](int x) {
        int y = 0;
        for (int b = 0; b < k; b++) {
            const int j = int(std::find(sorted, sorted + k, reg[b]) - sorted);  // canonical bit of q[b]
            if ((x >> j) & 1) y |= 1 << (k - 1 - b);
        }
        return y;
    };
    if (k == 2) code = kPhD2 + phase_pair(sorted[1], sorted[0]);
    if (k == 3) code = kPhD3 + phase_triple(sorted[2], sorted[1], sorted[0]);
    const int off = int(pool.size());
    for (int x = 0; x < D; x++)
        for (int xc = 0; xc < D; xc++) pool.push_back(src_pool[size_t(t.mat) + size_t(orig(x)) * D + orig(xc)]);
    return off;
}

}  // namespace

int plan_phases(const std::vector<TileOp>& ops, int m, bool c64, std::vector<double2>& pool,
                std::vector<TilePhase>& phases, std::vector<PhaseOp>& phase_ops) {
    const int N = int(ops.size());
    const int g = c64 ? 4 : 3;
    std::vector<uint32_t> T(N), S(N);
    for (int i = 0; i < N; i++) op_masks(ops[i], T[i], S[i]);
    // Matrices are copied out of the pool while it grows: read a snapshot.
    const std::vector<double2> src = pool;
    std::vector<char> done(N, 0);
    int left = N, count = 0;
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
        auto widen = [&](uint32_t R, uint32_t pool_bits, auto&& self) -> void {
            if (popcount32(R) >= kPhaseRegBits) {
                cands.push_back(R);
                return;
            }
            for (int b = 0; b < m; b++)
                if (((pool_bits >> b) & 1) && !((R >> b) & 1)) self(R | (1u << b), pool_bits, self);
        };
        for (uint32_t x : ready)
            if (x && popcount32(x) <= kPhaseRegBits) widen(x, all, widen);
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
        int Rb[kPhaseRegBits], nr = 0;
        for (int b = 0; b < m; b++)
            if ((R >> b) & 1) Rb[nr++] = b;
        // Slot bits: first one tile bit of each residue mod g (lowest first), so
        // the 2^g lanes of a shared-memory wavefront hit distinct bank groups;
        // then the other free bits ascending.
        std::vector<int> ord;
        std::vector<char> used(size_t(m), 0);
        for (int cls = 0; cls < g; cls++)
            for (int b = cls; b < m; b += g)
                if (!((R >> b) & 1)) {
                    ord.push_back(b);
                    used[size_t(b)] = 1;
                    break;
                }
        for (int b = 0; b < m; b++)
            if (!((R >> b) & 1) && !used[size_t(b)]) ord.push_back(b);
        TilePhase ph;
        ph.first_op = int(phase_ops.size());
        ph.nops = int(members.size());
        ph.nslot_bits = int(ord.size());
        for (int v = 0; v < kPhaseEntries; v++) {
            uint32_t o = 0;
            for (int i = 0; i < kPhaseRegBits; i++)
                if ((v >> i) & 1) o |= 1u << Rb[i];
            ph.rb[v] = o;
            ph.prb[v] = phase_swizzle(o, g);
        }
        for (size_t i = 0; i < ord.size(); i++) {
            ph.sb[i] = 1u << ord[i];
            ph.psb[i] = phase_swizzle(ph.sb[i], g);
        }
        for (int i : members) {
            const TileOp& t = ops[size_t(i)];
            PhaseOp p;
            switch (t.type) {
                case TileOp::kOne:
                case TileOp::kX: {
                    const int r = reg_of(Rb, __builtin_ctz(t.tbit));
                    p.code = (t.type == TileOp::kOne ? kPhOne : kPhX) + r;
                    p.mat = t.mat;
                    p.mask = S[size_t(i)] & ~t.tbit;
                    p.value = t.fixed;
                    break;
                }
                case TileOp::kSwap: {
                    const int lo = reg_of(Rb, __builtin_ctz(t.lowbit)), hi = reg_of(Rb, __builtin_ctz(t.highbit));
                    p.code = kPhSwap + phase_pair(hi, lo);
                    p.mask = S[size_t(i)] & ~(t.lowbit | t.highbit);
                    p.value = t.fixed;
                    break;
                }
                case TileOp::kDiagEntry:
                    p.code = kPhDiagEntry;
                    p.mat = t.mat;
                    p.mask = S[size_t(i)];
                    p.value = t.fixed;
                    break;
                case TileOp::kDiagFull:
                    p.code = kPhDiagFull;
                    p.mat = t.mat;
                    p.k = t.k;
                    for (int b = 0; b < t.k; b++) p.q[b] = uint8_t(t.q[b]);
                    break;
                case TileOp::kDense:
                    if (t.k == 1) {
                        p.code = kPhOne + reg_of(Rb, t.q[0]);
                        p.mat = t.mat;  // row-major 2x2: u00, u01, u10, u11
                    } else {
                        p.mat = canonical_dense(t, Rb, src, pool, p.code);
                    }
                    break;
                default: fail(kValueError, "tile operation without a phase form");
            }
            phase_ops.push_back(p);
            done[size_t(i)] = 1;
        }
        left -= int(members.size());
        phases.push_back(ph);
        count++;
    }
    return count;
}

namespace k {
namespace {

constexpr int kPhaseThreads = 256;

struct PhaseQubits {
    int m;
    int q[20];
};

constexpr int E = kPhaseEntries;

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

template <typename V, int T>
__device__ __forceinline__ void ph_one(V (&a)[E], const PhaseOp& op, const double2* __restrict__ pool,
                                       uint32_t base, const TilePhase* __restrict__ P) {
    const V u00 = dev::from_d2<V>(__ldg(pool + op.mat)), u01 = dev::from_d2<V>(__ldg(pool + op.mat + 1));
    const V u10 = dev::from_d2<V>(__ldg(pool + op.mat + 2)), u11 = dev::from_d2<V>(__ldg(pool + op.mat + 3));
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & (1 << T)) continue;
        const int w = v | (1 << T);
        if (op.mask && ((base | __ldg(&P->rb[v])) & op.mask) != op.value) continue;
        const V x = a[v], y = a[w];
        V p = dev::czero<V>(), q = dev::czero<V>();
        cmac(p, u00, x);
        cmac(p, u01, y);
        cmac(q, u10, x);
        cmac(q, u11, y);
        a[v] = p;
        a[w] = q;
    }
}

template <typename V, int T>
__device__ __forceinline__ void ph_x(V (&a)[E], const PhaseOp& op, uint32_t base, const TilePhase* __restrict__ P) {
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & (1 << T)) continue;
        const int w = v | (1 << T);
        if (op.mask && ((base | __ldg(&P->rb[v])) & op.mask) != op.value) continue;
        const V x = a[v];
        a[v] = a[w];
        a[w] = x;
    }
}

template <typename V, int H, int L>
__device__ __forceinline__ void ph_swap(V (&a)[E], const PhaseOp& op, uint32_t base, const TilePhase* __restrict__ P) {
#pragma unroll
    for (int v = 0; v < E; v++) {
        if (v & ((1 << H) | (1 << L))) continue;
        const int v01 = v | (1 << L), v10 = v | (1 << H);
        if (op.mask && ((base | __ldg(&P->rb[v01])) & op.mask) != op.value) continue;
        const V x = a[v01];
        a[v01] = a[v10];
        a[v10] = x;
    }
}

// Dense matrix of k = 2 or 3 qubits on register qubits Q[0] > ... > Q[k-1]
// (matrix index bit k-1-b on Q[b]), applied to every group of the other
// register qubits.  Rows are loaded one at a time; all groups' outputs are
// formed before any is written back.
template <typename V, int K, int Q0, int Q1, int Q2>
__device__ __forceinline__ void ph_dense(V (&a)[E], const PhaseOp& op, const double2* __restrict__ pool) {
    constexpr int D = 1 << K;
    constexpr int QM = (1 << Q0) | (1 << Q1) | (K == 3 ? (1 << Q2) : 0);
    constexpr int G = E / D;  // groups
    const double2* M = pool + op.mat;
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
        for (int c = 0; c < D; c++) mr[c] = dev::from_d2<V>(__ldg(M + r * D + c));
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

template <typename V>
__device__ __forceinline__ void ph_diag_entry(V (&a)[E], const PhaseOp& op, const double2* __restrict__ pool,
                                              uint32_t base, const TilePhase* __restrict__ P) {
    const V d = dev::from_d2<V>(__ldg(pool + op.mat));
#pragma unroll
    for (int v = 0; v < E; v++)
        if (((base | __ldg(&P->rb[v])) & op.mask) == op.value) a[v] = dev::cmul(a[v], d);
}

template <typename V>
__device__ __forceinline__ void ph_diag_full(V (&a)[E], const PhaseOp& op, const double2* __restrict__ pool,
                                             uint32_t base, const TilePhase* __restrict__ P) {
#pragma unroll
    for (int v = 0; v < E; v++) {
        const uint32_t full = base | __ldg(&P->rb[v]);
        uint32_t jj = 0;
#pragma unroll
        for (int b = 0; b < 8; b++)
            if (b < op.k) jj = (jj << 1) | ((full >> op.q[b]) & 1u);
        a[v] = dev::cmul(a[v], dev::from_d2<V>(__ldg(pool + op.mat + jj)));
    }
}

template <typename V>
__device__ __forceinline__ void ph_apply(V (&a)[E], const PhaseOp& op, const double2* __restrict__ pool,
                                         uint32_t base, const TilePhase* __restrict__ P) {
    switch (op.code) {
        case kPhOne + 0: ph_one<V, 0>(a, op, pool, base, P); break;
        case kPhOne + 1: ph_one<V, 1>(a, op, pool, base, P); break;
        case kPhOne + 2: ph_one<V, 2>(a, op, pool, base, P); break;
        case kPhX + 0: ph_x<V, 0>(a, op, base, P); break;
        case kPhX + 1: ph_x<V, 1>(a, op, base, P); break;
        case kPhX + 2: ph_x<V, 2>(a, op, base, P); break;
        case kPhD2 + phase_pair(1, 0): ph_dense<V, 2, 1, 0, 0>(a, op, pool); break;
        case kPhD2 + phase_pair(2, 0): ph_dense<V, 2, 2, 0, 0>(a, op, pool); break;
        case kPhD2 + phase_pair(2, 1): ph_dense<V, 2, 2, 1, 0>(a, op, pool); break;
        case kPhD3 + phase_triple(2, 1, 0): ph_dense<V, 3, 2, 1, 0>(a, op, pool); break;
        case kPhSwap + phase_pair(1, 0): ph_swap<V, 1, 0>(a, op, base, P); break;
        case kPhSwap + phase_pair(2, 0): ph_swap<V, 2, 0>(a, op, base, P); break;
        case kPhSwap + phase_pair(2, 1): ph_swap<V, 2, 1>(a, op, base, P); break;
#if DQ_PHASE_REG_BITS == 4
        case kPhOne + 3: ph_one<V, 3>(a, op, pool, base, P); break;
        case kPhX + 3: ph_x<V, 3>(a, op, base, P); break;
        case kPhD2 + phase_pair(3, 0): ph_dense<V, 2, 3, 0, 0>(a, op, pool); break;
        case kPhD2 + phase_pair(3, 1): ph_dense<V, 2, 3, 1, 0>(a, op, pool); break;
        case kPhD2 + phase_pair(3, 2): ph_dense<V, 2, 3, 2, 0>(a, op, pool); break;
        case kPhD3 + phase_triple(3, 1, 0): ph_dense<V, 3, 3, 1, 0>(a, op, pool); break;
        case kPhD3 + phase_triple(3, 2, 0): ph_dense<V, 3, 3, 2, 0>(a, op, pool); break;
        case kPhD3 + phase_triple(3, 2, 1): ph_dense<V, 3, 3, 2, 1>(a, op, pool); break;
        case kPhSwap + phase_pair(3, 0): ph_swap<V, 3, 0>(a, op, base, P); break;
        case kPhSwap + phase_pair(3, 1): ph_swap<V, 3, 1>(a, op, base, P); break;
        case kPhSwap + phase_pair(3, 2): ph_swap<V, 3, 2>(a, op, base, P); break;
#endif
        case kPhDiagEntry: ph_diag_entry<V>(a, op, pool, base, P); break;
        case kPhDiagFull: ph_diag_full<V>(a, op, pool, base, P); break;
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

template <typename V>
__global__ void __launch_bounds__(kPhaseThreads, kPhaseRegBits == 3 || sizeof(V) == 8 ? 2 : 1)
    k_tile_phased(V* __restrict__ s, int n, int m, PhaseQubits tq, const TilePhase* __restrict__ phases, int nphases,
                  const PhaseOp* __restrict__ ops, const double2* __restrict__ pool, uint64_t total_tiles) {
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
            const TilePhase* __restrict__ P = phases + p;
            const int nsb = __ldg(&P->nslot_bits), first = __ldg(&P->first_op), nops = __ldg(&P->nops);
            for (uint32_t sl = threadIdx.x; sl < slots; sl += blockDim.x) {
                uint32_t base = 0, pbase = 0;
                for (int i = 0; i < nsb; i++)
                    if ((sl >> i) & 1u) {
                        base |= __ldg(&P->sb[i]);
                        pbase ^= __ldg(&P->psb[i]);
                    }
                V a[E];
#pragma unroll
                for (int v = 0; v < E; v++) a[v] = tile[pbase ^ __ldg(&P->prb[v])];
                for (int o = 0; o < nops; o++) {
                    const PhaseOp op = ops[first + o];
                    ph_apply<V>(a, op, pool, base, P);
                }
#pragma unroll
                for (int v = 0; v < E; v++) tile[pbase ^ __ldg(&P->prb[v])] = a[v];
            }
            __syncthreads();
        }
        for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) gp[lo_tab[e & lmask] | hi_tab[e >> lb]] = tile[swz<V>(e)];
        __syncthreads();
    }
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

template <typename V>
void launch_phased(const Batch& b, const TilePass& hp, const TilePhase* phases, int nphases, const PhaseOp* ops,
                   const double2* pool) {
    const int m = int(hp.qubits.size());
    if (!phase_supported(m)) fail(kValueError, "tile pass too small or too large for register phases");
    PhaseQubits tq{};
    tq.m = m;
    for (int i = 0; i < m; i++) tq.q[i] = hp.qubits[size_t(i)];
    const size_t smem = tile_smem_bytes(m, sizeof(V) == 8);
    static size_t configured[2] = {0, 0};
    size_t& conf = configured[sizeof(V) == 8 ? 1 : 0];
    if (smem > conf) {
        cudaFuncSetAttribute(k_tile_phased<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(k_tile_phased<V>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
        conf = smem;
    }
    const uint64_t total = b.W << (b.n - m);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_phased<V>, kPhaseThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const uint64_t grid = std::min<uint64_t>(total, uint64_t(sm_count()) * per_sm);
    k_tile_phased<V><<<unsigned(grid), kPhaseThreads, smem, b.stream>>>(static_cast<V*>(b.amps), b.n, m, tq, phases,
                                                                         nphases, ops, pool, total);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("phased tile pass: ") + cudaGetErrorString(e));
}

}  // namespace

void tile_pass_phased(const Batch& b, const TilePass& host_pass, const TilePhase* phases_dev, int nphases,
                      const PhaseOp* ops_dev, const double2* pool_dev) {
    if (b.c64)
        launch_phased<float2>(b, host_pass, phases_dev, nphases, ops_dev, pool_dev);
    else
        launch_phased<double2>(b, host_pass, phases_dev, nphases, ops_dev, pool_dev);
}

}  // namespace k
}  // namespace dq

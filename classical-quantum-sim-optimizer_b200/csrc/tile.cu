// Shared-memory tile pass kernel and its host-side planner.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <set>

#include "common.hpp"
#include "cost.hpp"
#include "engine.hpp"
#include "tile.hpp"

namespace dq {

// ---------------------------------------------------------------------------
// Dense matrices of operations (qubits[0] = MSB of the matrix index)
// ---------------------------------------------------------------------------
namespace {

void op_matrix(const Operation& op, std::vector<uint64_t>& qs, std::vector<cplx>& mat) {
    qs.clear();
    auto controlled = [&](const std::vector<Control>& cs, int tk, auto&& inner) {
        // qubits = controls..., targets...; identity unless every control matches.
        for (auto& c : cs) qs.push_back(c.qubit);
        int k = int(qs.size()) + tk;
        int dim = 1 << k;
        mat.assign(size_t(dim) * dim, cplx(0));
        uint32_t want = 0;
        for (size_t i = 0; i < cs.size(); i++)
            if (cs[i].value) want |= 1u << (cs.size() - 1 - i);
        for (int r = 0; r < dim; r++) {
            uint32_t cr = uint32_t(r) >> tk;
            if (cr != want) {
                mat[size_t(r) * dim + r] = cplx(1);
                continue;
            }
            for (int c = 0; c < (1 << tk); c++) {
                int col = int((cr << tk) | uint32_t(c));
                mat[size_t(r) * dim + col] = inner(r & ((1 << tk) - 1), c);
            }
        }
    };
    switch (op.type) {
        case Operation::One:
            controlled(op.controls, 1, [&](int r, int c) { return op.m[r][c]; });
            qs.push_back(op.target);
            break;
        case Operation::X:
            controlled(op.controls, 1, [&](int r, int c) { return cplx(r != c ? 1.0 : 0.0); });
            qs.push_back(op.target);
            break;
        case Operation::Swap:
            controlled(op.controls, 2, [&](int r, int c) {
                int sw = ((c & 1) << 1) | ((c >> 1) & 1);
                return cplx(r == sw ? 1.0 : 0.0);
            });
            qs.push_back(op.a);
            qs.push_back(op.b);
            break;
        case Operation::Diagonal: {
            qs = op.qubits;
            size_t dim = op.values.size();
            mat.assign(dim * dim, cplx(0));
            for (size_t i = 0; i < dim; i++) mat[i * dim + i] = op.values[i];
            break;
        }
        case Operation::Dense:
            qs = op.qubits;
            mat = op.values;
            break;
        default: fail(kValueError, "operation has no matrix form");
    }
}

// Where op qubits `oq` sit in the index of block qubits `bq` (both MSB-first):
// ext[j] = op index of block index j, dep[v] = block bits of op index v.
struct Embedding {
    int dim = 0, odim = 0;
    uint32_t opmask = 0;
    std::vector<int> ext, dep;
    Embedding(const std::vector<uint64_t>& bq, const std::vector<uint64_t>& oq) {
        const int k = int(bq.size()), ko = int(oq.size());
        dim = 1 << k;
        odim = 1 << ko;
        std::vector<int> pos(static_cast<size_t>(ko));  // bit position (LSB = 0) of each op qubit in the block index
        for (int t = 0; t < ko; t++) {
            const int idx = int(std::find(bq.begin(), bq.end(), oq[size_t(t)]) - bq.begin());
            pos[size_t(t)] = k - 1 - idx;
            opmask |= 1u << pos[size_t(t)];
        }
        ext.assign(size_t(dim), 0);
        for (int j = 0; j < dim; j++)
            for (int t = 0; t < ko; t++) ext[size_t(j)] = (ext[size_t(j)] << 1) | ((j >> pos[size_t(t)]) & 1);
        dep.assign(size_t(odim), 0);
        for (int v = 0; v < odim; v++)
            for (int t = 0; t < ko; t++)
                if ((v >> (ko - 1 - t)) & 1) dep[size_t(v)] |= 1 << pos[size_t(t)];
    }
};

// The op matrix embedded on block qubits `bq` (identity on the others).
std::vector<cplx> embed(const std::vector<uint64_t>& bq, const std::vector<uint64_t>& oq,
                        const std::vector<cplx>& om) {
    const Embedding e(bq, oq);
    std::vector<cplx> out(size_t(e.dim) * e.dim, cplx(0));
    for (int r = 0; r < e.dim; r++) {
        const int rest = r & ~int(e.opmask), ro = e.ext[size_t(r)];
        for (int x = 0; x < e.odim; x++)
            out[size_t(r) * e.dim + (rest | e.dep[size_t(x)])] = om[size_t(ro) * e.odim + x];
    }
    return out;
}

// E = op matrix embedded on block qubits `bq` (MSB-first), then acc = E * acc.
void left_multiply(const std::vector<uint64_t>& bq, std::vector<cplx>& acc, const std::vector<uint64_t>& oq,
                   const std::vector<cplx>& om) {
    const Embedding e(bq, oq);
    const int dim = e.dim, odim = e.odim;
    std::vector<cplx> out(size_t(dim) * dim, cplx(0));
    for (int r = 0; r < dim; r++) {
        const int ro = e.ext[size_t(r)];
        const int rest = r & ~int(e.opmask);
        cplx* o = &out[size_t(r) * dim];
        for (int x = 0; x < odim; x++) {
            const cplx m = om[size_t(ro) * odim + x];
            if (m.re == 0.0 && m.im == 0.0) continue;
            const cplx* a = &acc[size_t(rest | e.dep[size_t(x)]) * dim];
            for (int c = 0; c < dim; c++) o[c] = o[c] + m * a[c];
        }
    }
    acc.swap(out);
}

bool is_identity_1(const cplx& v) { return v.re == 1.0 && v.im == 0.0; }

}  // namespace

namespace {

// The fused operation of `members` (in order) on qubits bq: dense, or diagonal
// when the product is.
Operation fused_operation(const std::vector<Operation>& ops, const std::vector<size_t>& members,
                          std::vector<uint64_t> bq) {
    std::sort(bq.begin(), bq.end(), std::greater<uint64_t>());
    const int dim = 1 << bq.size();
    std::vector<cplx> acc;
    std::vector<uint64_t> oq;
    std::vector<cplx> om;
    for (size_t mi : members) {
        op_matrix(ops[mi], oq, om);
        if (acc.empty())
            acc = embed(bq, oq, om);
        else
            left_multiply(bq, acc, oq, om);
    }
    Operation d;
    d.type = Operation::Dense;
    d.qubits = bq;
    d.values = acc;
    d.fused_count = 0;
    for (size_t mi : members) d.fused_count += ops[mi].fused_count;
    bool diag = true;
    for (int r = 0; r < dim && diag; r++)
        for (int c = 0; c < dim; c++)
            if (r != c && (acc[size_t(r) * dim + c].re != 0.0 || acc[size_t(r) * dim + c].im != 0.0)) {
                diag = false;
                break;
            }
    if (diag) {
        d.type = Operation::Diagonal;
        std::vector<cplx> dv(dim);
        for (int i = 0; i < dim; i++) dv[i] = acc[size_t(i) * dim + i];
        d.values = dv;
    }
    return d;
}

}  // namespace

std::vector<Operation> fuse_ops_lookahead(const std::vector<Operation>& ops, int width) {
    if (width <= 1) return ops;
    const size_t N = ops.size();
    std::vector<uint64_t> mask(N, 0);  // qubit masks (fused passes hold tile-local or global qubits < 64)
    for (size_t i = 0; i < N; i++)
        for (auto q : ops[i].touched()) {
            if (q >= 64) return fuse_ops(ops, width);
            mask[i] |= uint64_t(1) << q;
        }
    struct Blk {
        std::vector<size_t> members;
        uint64_t used;
    };
    // Ops absorbed by a block on qubit set S started at `first`: in order, an op
    // inside S joins unless an op left out earlier blocks one of its qubits.
    auto absorb = [&](const std::vector<char>& done, size_t first, uint64_t S, std::vector<size_t>& mem) {
        mem.clear();
        mem.push_back(first);
        uint64_t blocked = 0;
        for (size_t o = first + 1; o < N && (blocked & S) != S; o++) {
            if (done[o]) continue;
            if ((mask[o] & ~S) == 0 && (mask[o] & blocked) == 0)
                mem.push_back(o);
            else
                blocked |= mask[o];
        }
    };
    // The `keep` blocks that absorb the most operations among the 5-qubit sets
    // made of the first unfused operation's qubits and any of the next 12
    // distinct qubits (at most C(12, 4) = 495 sets; earliest set first on ties).
    auto candidates = [&](const std::vector<char>& done, size_t first, size_t keep) {
        std::vector<Blk> top;
        const int k0 = __builtin_popcountll(mask[first]);
        if (k0 > width) {  // wider than a block: stays on its own
            top.push_back({{first}, mask[first]});
            return top;
        }
        std::vector<int> cand;
        uint64_t seen = mask[first];
        for (size_t o = first + 1; o < N && cand.size() < 12; o++) {
            if (done[o]) continue;
            for (uint64_t fresh = mask[o] & ~seen; fresh && cand.size() < 12; fresh &= fresh - 1) {
                const int q = __builtin_ctzll(fresh);
                cand.push_back(q);
                seen |= uint64_t(1) << q;
            }
        }
        const int need = std::min<int>(width - k0, int(cand.size()));
        std::vector<int> pick(static_cast<size_t>(need));
        for (int i = 0; i < need; i++) pick[size_t(i)] = i;
        std::vector<size_t> mem;
        while (true) {
            uint64_t S = mask[first];
            for (int i = 0; i < need; i++) S |= uint64_t(1) << cand[size_t(pick[size_t(i)])];
            absorb(done, first, S, mem);
            uint64_t used = 0;
            for (size_t mi : mem) used |= mask[mi];
            bool dup = false;  // sets that absorb the same operations give the same block
            for (auto& t : top) dup = dup || t.members == mem;
            if (!dup) {
                auto at = std::find_if(top.begin(), top.end(), [&](const Blk& t) { return t.members.size() < mem.size(); });
                top.insert(at, Blk{mem, used});
                if (top.size() > keep) top.pop_back();
            }
            int i = need - 1;
            while (i >= 0 && pick[size_t(i)] == int(cand.size()) - need + i) i--;
            if (i < 0) break;
            pick[size_t(i)]++;
            for (int j = i + 1; j < need; j++) pick[size_t(j)] = pick[size_t(j - 1)] + 1;
        }
        return top;
    };
    // Beam search over block sequences: every level adds one block to each kept
    // sequence; sequences are ranked by the operations they cover, and the
    // first sequence that covers everything has the fewest blocks found.
    struct Seq {
        std::vector<char> done;
        std::vector<Blk> blocks;
        size_t covered = 0, first = 0;
    };
    constexpr size_t kBeam = 8, kBranch = 8;
    std::vector<Seq> beam(1);
    beam[0].done.assign(N, 0);
    std::vector<Blk> blocks;
    while (true) {
        bool finished = false;
        for (auto& q : beam) {
            while (q.first < N && q.done[q.first]) q.first++;
            if (q.first == N) {
                blocks = q.blocks;
                finished = true;
                break;
            }
        }
        if (finished || beam.empty()) break;
        std::vector<Seq> next;
        for (auto& q : beam)
            for (auto& b : candidates(q.done, q.first, kBranch)) {
                Seq c = q;
                for (size_t mi : b.members) c.done[mi] = 1;
                c.covered += b.members.size();
                c.blocks.push_back(b);
                next.push_back(std::move(c));
            }
        std::stable_sort(next.begin(), next.end(), [](const Seq& a, const Seq& b) { return a.covered > b.covered; });
        if (next.size() > kBeam) next.resize(kBeam);
        beam = std::move(next);
    }
    // Consecutive blocks whose qubits together fit in `width` run as one (the
    // fused sequence is a valid order, so their members simply concatenate).
    std::vector<Blk> merged;
    for (auto& b : blocks) {
        if (!merged.empty() && __builtin_popcountll(merged.back().used | b.used) <= width &&
            __builtin_popcountll(b.used) <= width) {
            merged.back().members.insert(merged.back().members.end(), b.members.begin(), b.members.end());
            merged.back().used |= b.used;
        } else {
            merged.push_back(std::move(b));
        }
    }
    std::vector<Operation> out;
    for (auto& b : merged) {
        if (b.members.size() == 1) {
            out.push_back(ops[b.members[0]]);
            continue;
        }
        std::vector<uint64_t> bq;
        for (uint64_t u = b.used; u; u &= u - 1) bq.push_back(uint64_t(__builtin_ctzll(u)));
        out.push_back(fused_operation(ops, b.members, bq));
    }
    return out;
}

std::vector<Operation> fuse_ops(const std::vector<Operation>& ops, int width) {
    if (width <= 1) return ops;
    const size_t N = ops.size();
    std::vector<std::vector<uint64_t>> qs(N);
    for (size_t i = 0; i < N; i++) qs[i] = ops[i].touched();
    uint64_t maxq = 0;
    for (auto& q : qs)
        for (auto v : q) maxq = std::max(maxq, v);
    std::vector<char> done(N, 0);
    std::vector<char> blocked(size_t(maxq) + 1, 0);
    std::vector<uint64_t> blocked_list;
    std::vector<Operation> out;
    for (size_t first = 0; first < N; first++) {
        if (done[first]) continue;
        if (qs[first].size() > size_t(width)) {
            done[first] = 1;
            out.push_back(ops[first]);
            continue;
        }
        std::vector<size_t> members{first};
        std::vector<uint64_t> bq = qs[first];
        done[first] = 1;
        // qubits blocked by an unfused operation that stays after this block
        for (auto q : blocked_list) blocked[size_t(q)] = 0;
        blocked_list.clear();
        for (size_t o = first + 1; o < N; o++) {
            if (done[o]) continue;
            bool touches_blocked = false;
            size_t uni = bq.size();
            for (auto q : qs[o]) {
                if (blocked[size_t(q)]) touches_blocked = true;
                if (std::find(bq.begin(), bq.end(), q) == bq.end()) uni++;
            }
            if (!touches_blocked && uni <= size_t(width)) {
                for (auto q : qs[o])
                    if (std::find(bq.begin(), bq.end(), q) == bq.end()) bq.push_back(q);
                members.push_back(o);
                done[o] = 1;
            } else {
                for (auto q : qs[o])
                    if (!blocked[size_t(q)]) {
                        blocked[size_t(q)] = 1;
                        blocked_list.push_back(q);
                    }
            }
            if (blocked_list.size() >= 64) break;
        }
        if (members.size() == 1) {
            out.push_back(ops[first]);
            continue;
        }
        std::sort(bq.begin(), bq.end(), std::greater<uint64_t>());
        const int dim = 1 << bq.size();
        std::vector<cplx> acc;
        std::vector<uint64_t> oq;
        std::vector<cplx> om;
        for (size_t mi : members) {
            op_matrix(ops[mi], oq, om);
            if (acc.empty())
                acc = embed(bq, oq, om);
            else
                left_multiply(bq, acc, oq, om);
        }
        Operation d;
        d.type = Operation::Dense;
        d.qubits = bq;
        d.values = acc;
        d.fused_count = 0;
        for (size_t mi : members) d.fused_count += ops[mi].fused_count;
        // Keep diagonal structure (cheaper kernels) when the product is diagonal.
        bool diag = true;
        for (int r = 0; r < dim && diag; r++)
            for (int c = 0; c < dim; c++)
                if (r != c && (acc[size_t(r) * dim + c].re != 0.0 || acc[size_t(r) * dim + c].im != 0.0)) {
                    diag = false;
                    break;
                }
        if (diag) {
            d.type = Operation::Diagonal;
            std::vector<cplx> dv(dim);
            for (int i = 0; i < dim; i++) dv[i] = acc[size_t(i) * dim + i];
            d.values = dv;
        }
        out.push_back(std::move(d));
    }
    return out;
}

// ---------------------------------------------------------------------------
// Fused tensor-core blocks
// ---------------------------------------------------------------------------
namespace {

// IEEE binary16 bits of v, rounded to nearest even (|v| below 65504).
uint16_t f16_rn(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    const uint16_t sign = uint16_t((u >> 16) & 0x8000u);
    const int e = int((u >> 23) & 0xFFu) - 127;
    const uint32_t m = (u & 0x7FFFFFu) | 0x800000u;  // 24-bit significand (normal inputs)
    if ((u & 0x7FFFFFFFu) == 0 || e < -25) return sign;
    if (e > 15) return uint16_t(sign | 0x7C00u);
    uint32_t q, rem, half;
    if (e < -14) {  // subnormal result: units of 2^-24
        const int shift = -(e + 1);
        q = m >> shift;
        rem = m & ((1u << shift) - 1u);
        half = 1u << (shift - 1);
    } else {  // normal: exponent field e + 15, 10 fraction bits
        q = (uint32_t(e + 15) << 10) | ((m & 0x7FFFFFu) >> 13);
        rem = m & 0x1FFFu;
        half = 0x1000u;
    }
    if (rem > half || (rem == half && (q & 1u))) q++;  // a carry moves into the exponent correctly
    return uint16_t(sign | q);
}

// Exact value of finite binary16 bits: a normal number's exponent and
// fraction move into binary32 fields; a subnormal is its fraction times 2^-24.
float f16_value(uint16_t h) {
    const uint32_t e = (h >> 10) & 0x1Fu, frac = h & 0x3FFu;
    float v;
    if (e) {
        const uint32_t bits = ((e + 112u) << 23) | (frac << 13);
        std::memcpy(&v, &bits, 4);
    } else {
        v = float(frac) * 0x1p-24f;
    }
    return (h & 0x8000u) ? -v : v;
}

}  // namespace

uint32_t fused_operand_offset(uint32_t packed) {
    const uint32_t col = packed >> 5, basis = packed & 31u;
    return (col >> 3) * 1024u + (col & 7u) * 128u + (((basis >> 2) ^ (col & 7u)) << 4) + (basis & 3u) * 4u;
}

namespace {

// Half-word offset of (row, k) in a K-major, 128-byte-swizzled operand with 64
// 16-bit K elements per row: row r at (r / 8) * 1024 + (r % 8) * 128 bytes, its
// 16-byte chunk index XORed with r % 8.
inline size_t sw128_half(int row, int k) {
    const size_t byte = size_t(row / 8) * 1024 + size_t(row % 8) * 128 + size_t(((k * 2) >> 4) ^ (row % 8)) * 16 +
                        size_t((k * 2) & 15);
    return byte / 2;
}

}  // namespace

namespace {

// Rank over GF(2) of up to 32-bit vectors.
int gf2_rank(std::vector<uint32_t> v) {
    int r = 0;
    for (int bit = 31; bit >= 0; bit--) {
        size_t piv = v.size();
        for (size_t i = size_t(r); i < v.size(); i++)
            if ((v[i] >> bit) & 1u) {
                piv = i;
                break;
            }
        if (piv == v.size()) continue;
        std::swap(v[size_t(r)], v[piv]);
        for (size_t i = 0; i < v.size(); i++)
            if (i != size_t(r) && ((v[i] >> bit) & 1u)) v[i] ^= v[size_t(r)];
        r++;
    }
    return r;
}

// The split's thread mapping (FusedPass::split_pos): lane bits 3 and 4 of a
// warp go to the first pair of local bits (4..11) whose banks in block 0's
// operand layout, with those of local bits 1..3, are independent.
void set_split_map(FusedPass& fp) {
    auto off = [&](uint32_t l) { return uint32_t(fp.in_lo[l & 63u] ^ fp.in_hi[l >> 6]); };
    auto bank = [&](int q) { return (off(1u << q) >> 2) & 31u; };
    int x = 4, y = 5;
    if (gf2_rank({bank(1), bank(2), bank(3), bank(4), bank(5)}) < 5) {
        bool found = false;
        for (int a = 4; a < kFusedM && !found; a++)
            for (int b = a + 1; b < kFusedM && !found; b++)
                if (gf2_rank({bank(1), bank(2), bank(3), bank(a), bank(b)}) == 5) {
                    x = a;
                    y = b;
                    found = true;
                }
    }
    int pos[kFusedM] = {0, 1, 2, 3, x, y};
    for (int q = 4, i = 6; q < kFusedM; q++)
        if (q != x && q != y) pos[i++] = q;
    for (int b = 0; b < 8; b++) fp.split_pos[b] = uint8_t(pos[b]);
    for (int k = 0; k < 16; k++) {
        uint32_t e = 0;
        for (int b = 0; b < 4; b++)
            if ((k >> b) & 1) e |= 1u << pos[8 + b];
        fp.split_q[k] = uint16_t(e);
        fp.split_qoff[k] = uint16_t(off(e));
    }
}

}  // namespace

FusedPass build_fused_pass(const std::vector<Operation>& pass_ops, const std::vector<int>& tile_qubits,
                           std::vector<FusedBlock>& blocks, std::vector<uint16_t>& upool) {
    FusedPass fp;
    fp.qubits = tile_qubits;
    fp.raw_ops = int(pass_ops.size());
    fp.first_block = int(blocks.size());
    const int m = int(tile_qubits.size());
    if (m != kFusedM) fail(kValueError, "fused passes hold exactly 12 tile qubits");
    std::vector<int> local(64, -1);
    for (int i = 0; i < m; i++) local[tile_qubits[i]] = i;
    // Block list: 5-qubit fusion, each block as (local qubits MSB-first, 32x32 matrix).
    struct Blk {
        int q[5];
        std::vector<cplx> u;
        int gates = 0;
    };
    std::vector<Blk> blk;
    for (const Operation& op : fuse_ops_lookahead(pass_ops, 5)) {
        std::vector<uint64_t> oq;
        std::vector<cplx> om;
        op_matrix(op, oq, om);
        std::vector<uint64_t> bq = oq;
        for (int i = 0; i < m && bq.size() < 5; i++) {
            uint64_t g = uint64_t(tile_qubits[i]);
            if (std::find(bq.begin(), bq.end(), g) == bq.end()) bq.push_back(g);
        }
        std::vector<cplx> acc = embed(bq, oq, om);
        Blk b;
        for (int t = 0; t < 5; t++) b.q[t] = local[bq[t]];
        b.u = std::move(acc);
        b.gates = std::max(1, op.fused_count);
        blk.push_back(std::move(b));
    }
    if (blk.empty()) {  // a pass of nothing but identities: one identity block
        Blk b;
        for (int t = 0; t < 5; t++) b.q[t] = 4 - t;
        b.u.assign(32 * 32, cplx(0));
        for (int i = 0; i < 32; i++) b.u[size_t(i) * 32 + i] = cplx(1);
        blk.push_back(std::move(b));
    }
    // Layout of block j: packed = (pext(l, other_j) << 5) | basis_j(l), basis MSB = q[0].
    auto layout = [&](const Blk& b, const std::vector<int>& oth, uint32_t l) {
        uint32_t basis = 0, col = 0;
        for (int t = 0; t < 5; t++) basis = (basis << 1) | ((l >> b.q[t]) & 1u);
        for (size_t t = 0; t < oth.size(); t++) col |= ((l >> oth[t]) & 1u) << t;
        return uint16_t((col << 5) | basis);
    };
    auto dep_basis = [&](const Blk& b, uint32_t basis) {
        uint32_t l = 0;
        for (int t = 0; t < 5; t++) l |= ((basis >> (4 - t)) & 1u) << b.q[t];
        return l;
    };
    auto dep_col = [&](const std::vector<int>& oth, uint32_t col) {
        uint32_t l = 0;
        for (size_t t = 0; t < oth.size(); t++) l |= ((col >> t) & 1u) << oth[t];
        return l;
    };
    // Bank-aware layouts.  The operand is stored 128-byte swizzled with 4-byte
    // complex entries (f16 re, im), so the bank of a store has bits (b0, b1,
    // b2^c0, b3^c1, b4^c2) of the block's basis (b) and column (c) index.
    // Across a warp, the readback of block j-1 varies the five qubits of its
    // column bits 0..4 (its TMEM lanes; local qubits 1..5 for the tile load).
    // Block j's basis and column bit order is chosen greedily so that those
    // five qubits reach five independent bank bits (one wavefront per warp):
    // lane qubits of the block at basis bits 0 and 1, lane qubits outside it
    // at column bits 0..2, the rest at basis bits 2..4.  Free column bits 0..4
    // then take qubits of block j+1 first (two of them are needed at its basis
    // bits 0 and 1).
    const size_t J = blk.size();
    std::vector<std::vector<int>> oth(J);
    // Qubits varying across a warp of the incoming stores: the tile load stores
    // pairs (l, l+1), so a warp's stores of one parity vary local qubits 1..5.
    uint32_t lanes = 0x3Eu;
    for (size_t j = 0; j < J; j++) {
        Blk& bj = blk[j];
        uint32_t bmask = 0, nmask = 0;
        for (int t = 0; t < 5; t++) bmask |= 1u << bj.q[t];
        if (j + 1 < J)
            for (int t = 0; t < 5; t++) nmask |= 1u << blk[j + 1].q[t];
        int bpos[5] = {-1, -1, -1, -1, -1};  // qubit at basis bit k
        int cpos[7] = {-1, -1, -1, -1, -1, -1, -1};
        uint32_t used = 0, reached = 0;  // reached bit k: bank bit k varies
        std::vector<int> lb, lc;
        for (int i = 0; i < m; i++)
            if ((lanes >> i) & 1u) ((bmask >> i) & 1u ? lb : lc).push_back(i);
        size_t bi = 0;
        for (int k = 0; k < 2 && bi < lb.size(); k++, bi++) {
            bpos[k] = lb[bi];
            used |= 1u << lb[bi];
            reached |= 1u << k;
        }
        size_t ci = 0;
        for (int k = 0; k < 3 && ci < lc.size(); k++, ci++) {
            cpos[k] = lc[ci];
            used |= 1u << lc[ci];
            reached |= 4u << k;
        }
        for (int k = 3; ci < lc.size(); k++, ci++) {  // more lane qubits than bank bits left: no bank
            cpos[k] = lc[ci];
            used |= 1u << lc[ci];
        }
        for (; bi < lb.size(); bi++) {
            int k = 2;
            while (k < 5 && (bpos[k] >= 0 || ((reached >> k) & 1u))) k++;
            if (k == 5) {
                k = 2;
                while (bpos[k] >= 0) k++;
            }
            bpos[k] = lb[bi];
            used |= 1u << lb[bi];
            reached |= 1u << k;
        }
        for (int t = 0; t < 5; t++)
            if (!((used >> bj.q[t]) & 1u))
                for (int k = 0; k < 5; k++)
                    if (bpos[k] < 0) {
                        bpos[k] = bj.q[t];
                        used |= 1u << bj.q[t];
                        break;
                    }
        // Column bits: lane qubits placed above, then qubits of the next block
        // (they become its basis bits), then the rest ascending.
        std::vector<int> rest;
        for (int i = 0; i < m; i++)
            if (!((bmask >> i) & 1u) && !((used >> i) & 1u)) rest.push_back(i);
        std::stable_sort(rest.begin(), rest.end(),
                         [&](int x, int y) { return ((nmask >> x) & 1u) > ((nmask >> y) & 1u); });
        size_t ri = 0;
        for (int k = 0; k < 7; k++)
            if (cpos[k] < 0) cpos[k] = rest[ri++];
        // Basis order q[t] = qubit at basis bit 4-t; permute the matrix to match.
        int old_bit[12];
        for (int t = 0; t < 5; t++) old_bit[bj.q[t]] = 4 - t;
        int perm[5];  // new basis bit k <- old basis bit perm[k]
        for (int k = 0; k < 5; k++) perm[k] = old_bit[bpos[k]];
        auto old_index = [&](int x) {
            int o = 0;
            for (int k = 0; k < 5; k++) o |= ((x >> k) & 1) << perm[k];
            return o;
        };
        std::vector<cplx> nu(32 * 32);
        for (int r = 0; r < 32; r++)
            for (int c = 0; c < 32; c++) nu[size_t(r) * 32 + c] = bj.u[size_t(old_index(r)) * 32 + old_index(c)];
        bj.u = std::move(nu);
        for (int t = 0; t < 5; t++) bj.q[t] = bpos[4 - t];
        oth[j].assign(cpos, cpos + 7);
        lanes = 0;
        for (int k = 0; k < 5; k++) lanes |= 1u << cpos[k];
    }
    // The last block's readback stores 8-byte FP32 entries, one half-warp at a
    // time: its column bits 0..3 vary across a half-warp.
    lanes &= ~(1u << oth[J - 1][4]);
    // Stage after the last block: natural index l lives at slot s(l) = l ^ h(l),
    // h copying lane qubits above bit 3 onto the bank bits 0..3 that the last
    // block's lanes leave constant (s is linear and invertible; a warp reading
    // consecutive l still covers every bank).  The sources are bits 4 and up,
    // so the slots of l and l ^ 1 stay the two halves of one 16-byte pair; when
    // bit 0 is a destination they may sit swapped, and the store phase reads
    // the pair at its 16-byte boundary and swaps it back.
    uint32_t hsrc[4] = {0, 0, 0, 0}, hdst[4] = {0, 0, 0, 0};
    int hn = 0;
    {
        std::vector<uint32_t> free_bits, high;
        for (uint32_t b = 0; b < 4; b++)
            if (!((lanes >> b) & 1u)) free_bits.push_back(b);
        for (uint32_t b = 4; b < 12; b++)
            if ((lanes >> b) & 1u) high.push_back(b);
        for (; hn < int(std::min(free_bits.size(), high.size())); hn++) {
            hsrc[hn] = high[size_t(hn)];
            hdst[hn] = free_bits[size_t(hn)];
        }
    }
    // Tables hold shared-memory byte offsets.  Both maps below are linear over
    // GF(2) in the local index, so parts of an index combine by XOR.
    auto stage_off = [&](uint32_t l) {
        uint32_t s = l;
        for (int i = 0; i < hn; i++) s ^= ((l >> hsrc[i]) & 1u) << hdst[i];
        return uint16_t(s * 8u);
    };
    auto operand_off = [&](const Blk& b, const std::vector<int>& oth, uint32_t l) {
        return uint16_t(fused_operand_offset(layout(b, oth, l)));
    };
    for (int e = 0; e < 64; e++) {
        fp.in_lo[e] = operand_off(blk[0], oth[0], uint32_t(e));
        fp.in_hi[e] = operand_off(blk[0], oth[0], uint32_t(e) << 6);
        fp.out_lo[e] = stage_off(uint32_t(e));
        fp.out_hi[e] = stage_off(uint32_t(e) << 6);
    }
    set_split_map(fp);
    for (size_t j = 0; j < blk.size(); j++) {
        FusedBlock d;
        std::memset(&d, 0, sizeof d);
        d.u_off = uint32_t(upool.size());
        d.last = j + 1 == blk.size() ? 1u : 0u;
        for (uint32_t bb = 0; bb < 32; bb++) {
            uint32_t l = dep_basis(blk[j], bb);
            d.next_b[bb] = d.last ? stage_off(l) : operand_off(blk[j + 1], oth[j + 1], l);
        }
        for (uint32_t c = 0; c < uint32_t(kFusedCols); c++) {
            uint32_t l = dep_col(oth[j], c);
            d.next_c[c] = d.last ? stage_off(l) : operand_off(blk[j + 1], oth[j + 1], l);
        }
        // Real 64x64 form [[Re, -Im], [Im, Re]] with rows 2b'+ri' and columns 2b+ri,
        // stored as the B operand (N = 64 output rows, K = 64 inputs, K-major,
        // 128-byte swizzled) in f16 hi and lo parts.
        std::vector<uint16_t> img(kFusedUHalves, 0);
        for (int bo = 0; bo < 32; bo++)
            for (int bi = 0; bi < 32; bi++) {
                const cplx v = blk[j].u[size_t(bo) * 32 + bi];
                const double e[2][2] = {{v.re, -v.im}, {v.im, v.re}};
                for (int ro = 0; ro < 2; ro++)
                    for (int ri = 0; ri < 2; ri++) {
                        const uint16_t hi = f16_rn(float(e[ro][ri]));
                        const uint16_t lo = f16_rn(float(e[ro][ri] - double(f16_value(hi))));
                        const size_t o = sw128_half(2 * bo + ro, 2 * bi + ri);
                        img[o] = hi;
                        img[kFusedUHalves / 2 + o] = lo;
                    }
            }
        upool.insert(upool.end(), img.begin(), img.end());
        blocks.push_back(d);
    }
    fp.nblocks = int(blk.size());
    for (const Blk& b : blk) {
        uint32_t mask = 0;
        for (int t = 0; t < 5; t++) mask |= 1u << b.q[t];
        fp.block_gates.push_back(b.gates);
        fp.block_masks.push_back(mask);
    }
    return fp;
}


FusedTma fused_tma_plan(const std::vector<int>& tile_qubits, int n, uint64_t states) {
    FusedTma t;
    const int m = int(tile_qubits.size());
    if (m != kFusedM || n < kFusedM || states == 0) return t;
    // Items in ascending bit order: tile chunks (<= 8 bits: a box side is at
    // most 256 elements) and the gaps between them.
    struct Item {
        int lo, bits;
        bool tile;
    };
    std::vector<Item> items;
    int pos = 0;
    for (int i = 0; i < m;) {
        int j = i;
        while (j + 1 < m && tile_qubits[size_t(j + 1)] == tile_qubits[size_t(j)] + 1) j++;
        const int a = tile_qubits[size_t(i)], e = tile_qubits[size_t(j)] + 1;
        if (a > pos) items.push_back({pos, a - pos, false});
        for (int c = a; c < e; c += 8) items.push_back({c, std::min(8, e - c), true});
        pos = e;
        i = j + 1;
    }
    uint64_t total = states << n;
    int total_bits = 0;
    while ((uint64_t(1) << total_bits) < total) total_bits++;
    int best_k = 0, best_cov = -1;
    for (int k = 1; k <= 5 && k <= int(items.size()); k++) {
        const Item& last = items[size_t(k - 1)];
        if (!last.tile) continue;
        // The last dimension's extent and coordinates must stay below 2^31.
        if (total_bits - last.lo > 31) continue;
        int cov = 0;
        for (int i = 0; i < k; i++)
            if (items[size_t(i)].tile) cov += items[size_t(i)].bits;
        if (cov > best_cov) {
            best_cov = cov;
            best_k = k;
        }
    }
    // At least 2 KiB per box (at most 16 boxes a tile).
    if (best_k == 0 || best_cov < 8) return t;
    t.ok = 1;
    t.dims = best_k;
    for (int i = 0; i < best_k; i++) {
        const Item& it = items[size_t(i)];
        t.lo[i] = it.lo;
        t.bits[i] = it.bits;
        t.box[i] = it.tile ? (1u << it.bits) : 1u;
        t.extent[i] = uint64_t(1) << it.bits;
    }
    t.extent[best_k - 1] = total >> t.lo[best_k - 1];
    t.copies = 1 << (kFusedM - best_cov);
    t.copy_bytes = uint32_t(8) << best_cov;
    for (int c = 0; c < t.copies; c++) {
        uint64_t extra = 0;
        for (int b = 0; best_cov + b < kFusedM; b++)
            if ((c >> b) & 1) extra |= uint64_t(1) << tile_qubits[size_t(best_cov + b)];
        t.copy_step[c] = int32_t(extra >> t.lo[best_k - 1]);
    }
    return t;
}

// ---------------------------------------------------------------------------
// Pass planner
// ---------------------------------------------------------------------------
namespace {

struct Dag {
    std::vector<std::vector<uint64_t>> qs;
    std::vector<uint64_t> mask;                  // qubits of each op as a bit mask (n <= 64)
    std::vector<std::vector<size_t>> per_qubit;  // op indices touching each qubit, in order
};

struct PlanState {
    std::vector<size_t> head;   // per qubit: position in per_qubit list
    std::vector<char> done;
    size_t first_open = 0;
};

bool ready(const Dag& g, const PlanState& s, size_t o) {
    for (auto q : g.qs[o])
        if (g.per_qubit[q][s.head[q]] != o) return false;
    return true;
}

void take(const Dag& g, PlanState& s, size_t o) {
    s.done[o] = 1;
    for (auto q : g.qs[o]) s.head[q]++;
    while (s.first_open < s.done.size() && s.done[s.first_open]) s.first_open++;
}

// The operation at the head of qubit q's list, SIZE_MAX when none is left.
size_t head_op(const Dag& g, const PlanState& s, size_t q) {
    return s.head[q] < g.per_qubit[q].size() ? g.per_qubit[q][s.head[q]] : SIZE_MAX;
}

// Absorbs every ready op inside T (bit mask) until nothing changes; appends
// them to `taken` and returns how many.  Only an op at the head of one of its
// qubits' lists can be ready, and taking an op moves only its own qubits'
// heads, so a worklist of heads finds the whole closure.
size_t closure(const Dag& g, PlanState& s, uint64_t T, std::vector<size_t>& taken, std::vector<size_t>& work) {
    work.clear();
    for (uint64_t r = T; r; r &= r - 1) {
        const size_t o = head_op(g, s, size_t(__builtin_ctzll(r)));
        if (o != SIZE_MAX) work.push_back(o);
    }
    size_t count = 0;
    while (!work.empty()) {
        const size_t o = work.back();
        work.pop_back();
        if (s.done[o] || (g.mask[o] & ~T) || !ready(g, s, o)) continue;
        take(g, s, o);
        taken.push_back(o);
        count++;
        for (auto q : g.qs[o])
            if (head_op(g, s, q) != SIZE_MAX) work.push_back(head_op(g, s, q));
    }
    return count;
}

// Reverts the ops in `taken` (first_open is restored by the caller).
void untake(const Dag& g, PlanState& s, const std::vector<size_t>& taken) {
    for (size_t i = taken.size(); i-- > 0;) {
        s.done[taken[i]] = 0;
        for (auto q : g.qs[taken[i]]) s.head[q]--;
    }
}

// What a pass's tile qubits may be: m of them, qubits 0..pinned-1 always, and a
// spread (below) of at most max_spread.
//
// The tiles a pass has in flight at once differ in the lowest `inflight_bits`
// qubits outside T, so together they read contiguous runs of 2^c amplitudes,
// c the lowest qubit neither in T nor among those; the high tile qubits
// scatter those runs.  The spread, in quarters, is 4 per tile qubit at or above
// spread_bit + 4, 3 per tile qubit in [spread_bit, spread_bit + 4), less 12
// per tile qubit that lengthens the runs (those in [pinned, c)).
struct TileShape {
    int m, n, pinned, spread_bit, max_spread, inflight_bits;
    size_t max_ops = 0;  // operations per pass (0: no limit)
    int spread(uint64_t T) const {
        if (spread_bit >= 64) return 0;
        const uint64_t hi = T >> spread_bit;
        const int top = __builtin_popcountll(hi >> 4), mid = __builtin_popcountll(hi & 15);
        int run_bits = 0, outside = 0;
        for (int q = 0; q < n; q++) {
            if ((T >> q) & 1) {
                run_bits += q >= pinned ? 1 : 0;
            } else if (++outside > inflight_bits) {
                break;
            }
        }
        return 4 * top + 3 * mid - 12 * run_bits;
    }
};

// Reused buffers of one thread's grow() calls.
struct GrowScratch {
    std::vector<size_t> cands, trial, work;
    std::vector<uint64_t> tried;
};

// Grows T from a seed op: the pinned qubits and the seed's, then, while T has
// room, the new qubits of one ready op at a time.  Of the ready ops whose
// qubits fit, the one whose new qubits let the most ops in per added qubit is
// chosen (fewer new qubits, then the earliest op, on ties).  Returns the ops
// absorbed, in the order taken, and T; `s` is left as it was.
size_t grow(const Dag& g, PlanState& s, size_t seed, const TileShape& sh, bool lookahead, uint64_t& T,
            std::vector<size_t>& taken, GrowScratch& x) {
    const int m = sh.m, n = sh.n;
    const size_t first_open = s.first_open;
    taken.clear();
    T = (sh.pinned >= 64 ? ~uint64_t(0) : (uint64_t(1) << sh.pinned) - 1) | g.mask[seed];
    if (n < 64) T &= (uint64_t(1) << n) - 1;
    int size = __builtin_popcountll(T);
    closure(g, s, T, taken, x.work);
    while (size < m) {
        x.cands.clear();
        for (size_t q = 0; q < size_t(n); q++) {
            const size_t o = head_op(g, s, q);
            if (o != SIZE_MAX && ready(g, s, o)) x.cands.push_back(o);
        }
        std::sort(x.cands.begin(), x.cands.end());
        x.cands.erase(std::unique(x.cands.begin(), x.cands.end()), x.cands.end());
        size_t best = SIZE_MAX;
        size_t best_gain = 0;
        int best_new = 1;
        x.tried.clear();  // new-qubit sets already scored
        for (size_t o : x.cands) {
            const uint64_t fresh = g.mask[o] & ~T;
            const int nw = __builtin_popcountll(fresh);
            if (nw == 0 || size + nw > m) continue;
            if (std::find(x.tried.begin(), x.tried.end(), fresh) != x.tried.end()) continue;
            x.tried.push_back(fresh);
            if (sh.spread(T | fresh) > sh.max_spread) continue;
            size_t gain = 0;
            if (lookahead) {
                const size_t fo = s.first_open;
                x.trial.clear();
                gain = closure(g, s, T | fresh, x.trial, x.work);
                untake(g, s, x.trial);
                s.first_open = fo;
            }
            // gain / nw > best_gain / best_new, or equal with fewer new qubits
            const size_t lhs = gain * size_t(best_new), rhs = best_gain * size_t(nw);
            if (best == SIZE_MAX || lhs > rhs || (lhs == rhs && nw < best_new)) {
                best = o;
                best_gain = gain;
                best_new = nw;
            }
        }
        if (best == SIZE_MAX) break;
        T |= g.mask[best];
        size = __builtin_popcountll(T);
        closure(g, s, T, taken, x.work);
    }
    untake(g, s, taken);
    s.first_open = first_open;
    // A depth limit keeps the first operations taken (a dependency-closed prefix).
    if (sh.max_ops && taken.size() > sh.max_ops) taken.resize(sh.max_ops);
    return taken.size();
}

// One pass of a plan: its tile qubits (before padding) and the ops it takes.
struct PassChoice {
    uint64_t T = 0;
    std::vector<size_t> taken;
};

// Chooses the passes.  Each pass is grown from one of the first `seeds` ready
// ops by either growth rule (fewest new qubits; most ops let in per new
// qubit); a beam of `beam` partial plans, ranked by the ops they cover after
// the same number of passes, keeps the best extensions, and the first plan to
// cover every op wins (beam 1: the single best pass each time).
std::vector<PassChoice> choose_passes(const Dag& g, const TileShape& sh, int seeds, int beam) {
    const size_t N = g.qs.size();
    struct Node {
        PlanState s;
        size_t covered = 0;
        std::vector<int> chain;  // indices into `arena`
    };
    std::vector<PassChoice> arena;
    std::vector<Node> nodes(1);
    nodes[0].s.head.assign(size_t(sh.n), 0);
    nodes[0].s.done.assign(N, 0);
    while (true) {
        for (const Node& nd : nodes)
            if (nd.s.first_open >= N) {
                std::vector<PassChoice> out;
                for (int i : nd.chain) out.push_back(arena[size_t(i)]);
                return out;
            }
        struct Cand {
            size_t node, covered;
            PassChoice pc;
        };
        // Each node's extensions, distinct by tile qubits (the same qubits from
        // the same state take the same ops); nodes expand on separate threads.
        std::vector<std::vector<Cand>> per_node(nodes.size());
        auto expand = [&](size_t ni) {
            Node& nd = nodes[ni];
            std::vector<Cand>& out = per_node[ni];
            uint64_t T = 0;
            std::vector<size_t> taken;
            GrowScratch x;
            std::vector<size_t> seed_ops;
            for (size_t o = nd.s.first_open; o < N && int(seed_ops.size()) < seeds; o++)
                if (!nd.s.done[o] && ready(g, nd.s, o)) seed_ops.push_back(o);
            for (int la = 0; la < 2; la++)
                for (size_t sd : seed_ops) {
                    const size_t c = grow(g, nd.s, sd, sh, la == 1, T, taken, x);
                    bool dup = false;
                    for (size_t k = 0; k < out.size() && !dup; k++) dup = out[k].pc.T == T;
                    if (!dup) out.push_back(Cand{ni, nd.covered + c, PassChoice{T, taken}});
                }
        };
        if (nodes.size() > 1)
            parallel_for(nodes.size(), expand);
        else
            expand(0);
        std::vector<Cand> cands;
        for (auto& v : per_node)
            for (auto& c : v) cands.push_back(std::move(c));
        std::stable_sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.covered > y.covered; });
        if (cands.size() > size_t(beam)) cands.resize(size_t(beam));
        std::vector<Node> next;
        for (Cand& c : cands) {
            Node nd = nodes[c.node];
            for (size_t o : c.pc.taken) take(g, nd.s, o);
            nd.covered = c.covered;
            nd.chain.push_back(int(arena.size()));
            arena.push_back(std::move(c.pc));
            next.push_back(std::move(nd));
        }
        nodes = std::move(next);
    }
}

TileOp lower_tile_op(const Operation& op, const std::vector<int>& local, std::vector<double2>& pool,
                     std::vector<TileOp>& out) {
    TileOp t;
    std::memset(&t, 0, sizeof t);
    t.ngates = op.fused_count;
    auto L = [&](uint64_t q) { return local[q]; };
    auto set_ins = [&](std::vector<int> pos) {
        std::sort(pos.begin(), pos.end());
        t.nins = int(pos.size());
        for (size_t i = 0; i < pos.size(); i++) t.ins[i] = pos[i];
    };
    auto d2 = [](cplx c) { return make_double2(c.re, c.im); };
    switch (op.type) {
        case Operation::One:
        case Operation::X: {
            t.type = op.type == Operation::One ? TileOp::kOne : TileOp::kX;
            std::vector<int> pos{L(op.target)};
            for (auto& c : op.controls) {
                pos.push_back(L(c.qubit));
                if (c.value) t.fixed |= 1u << L(c.qubit);
            }
            set_ins(pos);
            t.tbit = 1u << L(op.target);
            t.mat = int(pool.size());
            if (op.type == Operation::One) {
                pool.push_back(d2(op.m[0][0]));
                pool.push_back(d2(op.m[0][1]));
                pool.push_back(d2(op.m[1][0]));
                pool.push_back(d2(op.m[1][1]));
            }
            out.push_back(t);
            break;
        }
        case Operation::Swap: {
            t.type = TileOp::kSwap;
            std::vector<int> pos{L(op.a), L(op.b)};
            for (auto& c : op.controls) {
                pos.push_back(L(c.qubit));
                if (c.value) t.fixed |= 1u << L(c.qubit);
            }
            set_ins(pos);
            int lo = std::min(L(op.a), L(op.b)), hi = std::max(L(op.a), L(op.b));
            t.lowbit = 1u << lo;
            t.highbit = 1u << hi;
            out.push_back(t);
            break;
        }
        case Operation::Diagonal: {
            const int kq = int(op.qubits.size());
            std::vector<int> nontrivial;
            for (int j = 0; j < (1 << kq); j++)
                if (!is_identity_1(op.values[j])) nontrivial.push_back(j);
            if (nontrivial.empty()) break;
            std::vector<int> lq;
            for (auto q : op.qubits) lq.push_back(L(q));
            if (int(nontrivial.size()) * 2 <= (1 << kq)) {
                for (int j : nontrivial) {
                    TileOp e;
                    std::memset(&e, 0, sizeof e);
                    e.type = TileOp::kDiagEntry;
                    e.ngates = op.fused_count;
                    std::vector<int> pos(lq);
                    std::sort(pos.begin(), pos.end());
                    e.nins = int(pos.size());
                    for (size_t i = 0; i < pos.size(); i++) e.ins[i] = pos[i];
                    for (int b = 0; b < kq; b++)
                        if ((j >> (kq - 1 - b)) & 1) e.fixed |= 1u << lq[b];
                    e.mat = int(pool.size());
                    pool.push_back(d2(op.values[j]));
                    out.push_back(e);
                }
            } else {
                t.type = TileOp::kDiagFull;
                t.k = kq;
                for (int b = 0; b < kq; b++) t.q[b] = lq[b];
                t.mat = int(pool.size());
                for (auto& v : op.values) pool.push_back(d2(v));
                out.push_back(t);
            }
            break;
        }
        case Operation::Dense: {
            t.type = TileOp::kDense;
            t.k = int(op.qubits.size());
            std::vector<int> lq;
            for (auto q : op.qubits) lq.push_back(L(q));
            for (int b = 0; b < t.k; b++) t.q[b] = lq[b];
            set_ins(lq);
            for (int j = 0; j < (1 << t.k); j++) {
                uint32_t o = 0;
                for (int b = 0; b < t.k; b++)
                    if ((j >> (t.k - 1 - b)) & 1) o |= 1u << lq[b];
                t.offs[j] = o;
            }
            t.mat = int(pool.size());
            for (auto& v : op.values) pool.push_back(d2(v));
            out.push_back(t);
            break;
        }
        default: fail(kValueError, "operation cannot run inside a tile pass");
    }
    return t;
}

}  // namespace

std::vector<int> fused_caps(int n, bool wide) {
    std::vector<int> caps{kFusedMaxSpread};
    if (4 * (n - kFusedSpreadBit) - 4 > kFusedMaxSpread) {
        caps.push_back(-1);
        caps.push_back(kFusedMaxSpread - 4);
        if (wide)
            for (int c : {kFusedMaxSpread - 8, kFusedMaxSpread + 4, kFusedMaxSpread + 8})
                if (c >= 0 && (c <= kFusedMaxSpread || 4 * (n - kFusedSpreadBit) - 4 > c)) caps.push_back(c);
    }
    return caps;
}

FusedPortfolio fused_portfolio(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                               const TilePlanOptions& base, const std::vector<int>& caps) {
    TilePlanOptions o = base;
    o.m = kFusedM;
    o.keep_raw = true;
    o.pinned_low = kFusedPinned;
    o.spread_bit = kFusedSpreadBit;
    o.beam = kPlanBeam;
    o.model = nullptr;
    o.chosen_widths = nullptr;
    FusedPortfolio pf;
    pf.n = n;
    pf.caps = caps;
    pf.plans.resize(caps.size());
    parallel_for(caps.size(), [&](size_t i) {
        TilePlanOptions oi = o;
        oi.max_spread = caps[i];
        std::vector<double2> unused;
        pf.plans[i] = plan_tiles(ops, begin, end, n, oi, &unused);
    });
    // The plans share passes (same tile qubits, same operations): each distinct
    // pass is fused into blocks once, all of them on pooled workers.
    std::map<std::pair<std::vector<int>, std::vector<size_t>>, size_t> slot_of;
    std::vector<const TilePass*> distinct;
    pf.slots.resize(pf.plans.size());
    for (size_t i = 0; i < pf.plans.size(); i++)
        for (const TilePass& p : pf.plans[i]) {
            auto it = slot_of.emplace(std::make_pair(p.qubits, p.op_index), distinct.size()).first;
            if (it->second == distinct.size()) distinct.push_back(&p);
            pf.slots[i].push_back(it->second);
        }
    pf.built.resize(distinct.size());
    parallel_for(distinct.size(), [&](size_t k) {
        BuiltFusedPass& b = pf.built[k];
        b.fp = build_fused_pass(distinct[k]->raw, distinct[k]->qubits, b.blocks, b.upool);
    });
    const TileShape sh{kFusedM, n, kFusedPinned, kFusedSpreadBit, INT_MAX, o.inflight_bits};
    pf.rule_cost.assign(pf.plans.size(), 0.0);
    for (size_t i = 0; i < pf.plans.size(); i++) {
        double cost = kFusedPassCostBlocks * double(pf.plans[i].size());
        for (size_t k = 0; k < pf.plans[i].size(); k++) {
            uint64_t T = 0;
            for (int q : pf.plans[i][k].qubits) T |= uint64_t(1) << q;
            const int spread = sh.spread(T);
            cost += pf.built[pf.slots[i][k]].fp.nblocks + (spread > kFusedMaxSpread + 4   ? kFusedSpreadCostBlocks[1]
                                                           : spread > kFusedMaxSpread ? kFusedSpreadCostBlocks[0]
                                                                                      : 0.0);
        }
        pf.rule_cost[i] = cost;
        if (i == 0 || cost < pf.rule_cost[pf.rule_choice]) pf.rule_choice = i;
    }
    return pf;
}

std::vector<BuiltFusedPass> take_fused_plan(FusedPortfolio& pf, size_t i) {
    std::vector<BuiltFusedPass> out(pf.plans[i].size());
    for (size_t k = 0; k < out.size(); k++) {
        const size_t slot = pf.slots[i][k];
        out[k].fp = pf.built[slot].fp;
        out[k].blocks = pf.built[slot].blocks;
        out[k].upool = pf.built[slot].upool;
        out[k].src = std::move(pf.plans[i][k]);
    }
    return out;
}

std::vector<BuiltFusedPass> plan_fused(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                                       const TilePlanOptions& base) {
    FusedPortfolio pf = fused_portfolio(ops, begin, end, n, base, fused_caps(n, false));
    return take_fused_plan(pf, pf.rule_choice);
}

void lower_pass_ops(const std::vector<Operation>& raw, const std::vector<int>& tile_qubits, int n, int width,
                    std::vector<double2>& pool, std::vector<TileOp>& out) {
    std::vector<int> local(size_t(n), -1);
    for (size_t i = 0; i < tile_qubits.size(); i++) local[size_t(tile_qubits[i])] = int(i);
    for (auto& op : fuse_ops(raw, width)) lower_tile_op(op, local, pool, out);
}

std::vector<TilePass> plan_tiles(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                                 const TilePlanOptions& opt, std::vector<double2>* pool) {
    std::vector<TilePass> passes;
    const size_t N = end - begin;
    if (N == 0) return passes;
    // A pass holds every qubit of each of its operations.
    int widest = 1;
    for (size_t i = begin; i < end; i++) widest = std::max(widest, int(ops[i].touched().size()));
    const int pinned = std::min(std::max(opt.pinned_low, 0), n);
    const int m = std::min(std::max(opt.m, widest + pinned), n);
    if (n > 64) fail(kValueError, "tile passes take at most 64 qubits");
    Dag g;
    g.qs.resize(N);
    g.mask.assign(N, 0);
    g.per_qubit.assign(n, {});
    for (size_t i = 0; i < N; i++) {
        g.qs[i] = ops[begin + i].touched();
        for (auto q : g.qs[i]) {
            g.per_qubit[q].push_back(i);
            g.mask[i] |= uint64_t(1) << q;
        }
    }
    const int beam = N > kPlanBeamMaxOps ? 1 : std::max(1, opt.beam);
    // A seed's own qubits are always allowed; the cap applies to the rest.
    TileShape sh{m, n, pinned, std::max(opt.spread_bit, 0), opt.max_spread >= 0 ? opt.max_spread : INT_MAX,
                 std::max(opt.inflight_bits, 0), size_t(std::max(opt.max_pass_ops, 0))};
    const std::vector<PassChoice> chosen = choose_passes(g, sh, std::max(1, opt.seeds), beam);
    for (const PassChoice& pc : chosen) {
        std::vector<char> inT(size_t(n), 0);
        for (int q = 0; q < n; q++) inT[size_t(q)] = char((pc.T >> q) & 1);
        std::vector<size_t> taken = pc.taken;
        // Circuit order is a valid order for any set of ops, and the block
        // fusion below starts each block at the first op left.
        std::sort(taken.begin(), taken.end());
        // pad T to m qubits with the lowest free qubits (longer contiguous rows)
        int size = 0;
        for (int q = 0; q < n; q++) size += inT[q];
        for (int q = 0; q < n && size < m; q++)
            if (!inT[q]) {
                inT[q] = 1;
                size++;
            }
        TilePass p;
        for (int q = 0; q < n; q++)
            if (inT[q]) p.qubits.push_back(q);
        std::vector<int> local(n, -1);
        for (size_t i = 0; i < p.qubits.size(); i++) local[p.qubits[i]] = int(i);
        std::vector<Operation> pass_ops;
        for (size_t o : taken) pass_ops.push_back(ops[begin + o]);
        p.raw_ops = int(pass_ops.size());
        for (size_t o : taken) p.op_index.push_back(begin + o);
        if (opt.keep_raw) {
            p.raw = std::move(pass_ops);
            passes.push_back(std::move(p));
            continue;
        }
        int width = opt.fuse;
        if (opt.model) {
            // The cost model judges each candidate width by its lowered operations.
            double best = 1e300;
            for (int w = 1; w <= kTileMaxDense; w++) {
                std::vector<double2> scratch;
                std::vector<TileOp> cand;
                for (auto& op : fuse_ops(pass_ops, w)) lower_tile_op(op, local, scratch, cand);
                double cost = opt.model->predict_ops(cand, int(p.qubits.size()), opt.c64);
                if (cost < best) {
                    best = cost;
                    width = w;
                }
            }
        }
        if (opt.chosen_widths) opt.chosen_widths->push_back(width);
        std::vector<Operation> fused = fuse_ops(pass_ops, width);
        for (auto& op : fused) lower_tile_op(op, local, *pool, p.ops);
        passes.push_back(std::move(p));
    }
    return passes;
}

// ---------------------------------------------------------------------------
// Kernel
// ---------------------------------------------------------------------------
namespace k {
namespace {

constexpr int kTileThreads = 256;

struct TileQubits {
    int m;
    int q[20];
};

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

// Insertion positions of one operation, held in registers for its whole loop.
struct Ins {
    int n;
    int p[7];
};

__device__ __forceinline__ Ins load_ins(const TileOp& op) {
    Ins s;
    s.n = op.nins;
#pragma unroll
    for (int t = 0; t < 7; t++) s.p[t] = op.ins[t];
    return s;
}

__device__ __forceinline__ uint32_t expand_ins(uint32_t j, const Ins& s) {
#pragma unroll
    for (int t = 0; t < 7; t++) {
        if (t < s.n) {
            uint32_t low = (1u << s.p[t]) - 1;
            j = (j & low) | ((j & ~low) << 1);
        }
    }
    return j;
}

// acc += m * v as four fused multiply-adds (the products are not rounded
// before the sum): a third fewer FP64 instructions than a rounded product plus
// a separate sum.
__device__ __forceinline__ void tmac(double2& acc, double2 m, double2 v) {
    acc.x = fma(m.x, v.x, acc.x);
    acc.x = fma(-m.y, v.y, acc.x);
    acc.y = fma(m.x, v.y, acc.y);
    acc.y = fma(m.y, v.x, acc.y);
}
__device__ __forceinline__ void tmac(float2& acc, float2 m, float2 v) {
    acc.x = fmaf(m.x, v.x, acc.x);
    acc.x = fmaf(-m.y, v.y, acc.x);
    acc.y = fmaf(m.x, v.y, acc.y);
    acc.y = fmaf(m.y, v.x, acc.y);
}

// 1- and 2-qubit dense matrices: matrix and offsets in registers, rows fully
// unrolled so the 4 (16) complex products of a group are independent.
template <typename V, int K>
__device__ void tile_dense_small(V* __restrict__ tile, const TileOp& op, int m, const double2* __restrict__ pool) {
    constexpr int D = 1 << K;
    const uint32_t items = 1u << (m - K);
    V M[D * D];
#pragma unroll
    for (int i = 0; i < D * D; i++) M[i] = dev::from_d2<V>(__ldg(pool + op.mat + i));
    uint32_t off[D];
#pragma unroll
    for (int c = 0; c < D; c++) off[c] = op.offs[c];
    const Ins ins = load_ins(op);
    for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
        const uint32_t base = expand_ins(j, ins);
        V v[D];
#pragma unroll
        for (int c = 0; c < D; c++) v[c] = tile[base | off[c]];
#pragma unroll
        for (int r = 0; r < D; r++) {
            V acc = dev::czero<V>();
#pragma unroll
            for (int c = 0; c < D; c++) tmac(acc, M[r * D + c], v[c]);
            tile[base | off[r]] = acc;
        }
    }
}

template <typename V, int K>
__device__ void tile_dense(V* __restrict__ tile, const TileOp& op, int m, const double2* __restrict__ pool) {
    constexpr int D = 1 << K;
    const uint32_t items = 1u << (m - K);
    const double2* mat = pool + op.mat;
    uint32_t off[D];
#pragma unroll
    for (int c = 0; c < D; c++) off[c] = op.offs[c];
    const Ins ins = load_ins(op);
    for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
        const uint32_t base = expand_ins(j, ins);
        V v[D];
#pragma unroll
        for (int c = 0; c < D; c++) v[c] = tile[base | off[c]];
#pragma unroll 1
        for (int r = 0; r < D; r++) {
            V acc = dev::czero<V>();
#pragma unroll
            for (int c = 0; c < D; c++) tmac(acc, dev::from_d2<V>(__ldg(mat + r * D + c)), v[c]);
            tile[base | op.offs[r]] = acc;  // row offset from the (cached) descriptor: no dynamic register index
        }
    }
}

template <typename V>
__device__ void tile_apply(V* __restrict__ tile, const TileOp& op, int m, const double2* __restrict__ pool) {
    switch (op.type) {
        case TileOp::kOne:
        case TileOp::kX: {
            const Ins ins = load_ins(op);
            const uint32_t items = 1u << (m - ins.n);
            const uint32_t fixed = op.fixed, tbit = op.tbit;
            const bool is_x = op.type == TileOp::kX;
            V u00 = dev::czero<V>(), u01 = u00, u10 = u00, u11 = u00;
            if (!is_x) {
                u00 = dev::from_d2<V>(__ldg(pool + op.mat));
                u01 = dev::from_d2<V>(__ldg(pool + op.mat + 1));
                u10 = dev::from_d2<V>(__ldg(pool + op.mat + 2));
                u11 = dev::from_d2<V>(__ldg(pool + op.mat + 3));
            }
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i0 = expand_ins(j, ins) | fixed, i1 = i0 | tbit;
                V a = tile[i0], b = tile[i1];
                if (is_x) {
                    tile[i0] = b;
                    tile[i1] = a;
                } else {
                    V p = dev::czero<V>(), q = dev::czero<V>();
                    tmac(p, u00, a);
                    tmac(p, u01, b);
                    tmac(q, u10, a);
                    tmac(q, u11, b);
                    tile[i0] = p;
                    tile[i1] = q;
                }
            }
            break;
        }
        case TileOp::kDiagEntry: {
            const Ins ins = load_ins(op);
            const uint32_t items = 1u << (m - ins.n);
            const uint32_t fixed = op.fixed;
            const V v = dev::from_d2<V>(__ldg(pool + op.mat));
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i = expand_ins(j, ins) | fixed;
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
            const Ins ins = load_ins(op);
            const uint32_t items = 1u << (m - ins.n);
            const uint32_t fixed = op.fixed, lo = op.lowbit, hi = op.highbit;
            for (uint32_t j = threadIdx.x; j < items; j += blockDim.x) {
                const uint32_t i = expand_ins(j, ins) | fixed;
                V a = tile[i | lo];
                tile[i | lo] = tile[i | hi];
                tile[i | hi] = a;
            }
            break;
        }
        case TileOp::kDense:
            switch (op.k) {
                case 1: tile_dense_small<V, 1>(tile, op, m, pool); break;
                case 2: tile_dense_small<V, 2>(tile, op, m, pool); break;
                case 3: tile_dense<V, 3>(tile, op, m, pool); break;
            }
            break;
    }
}

template <typename V, bool TIMED>
__global__ void __launch_bounds__(kTileThreads, 2) k_tile(V* __restrict__ s, int n, int m, TileQubits tq,
                                                       const TileOp* __restrict__ ops, int nops,
                                                       const double2* __restrict__ pool, uint64_t total_tiles,
                                                       unsigned long long* __restrict__ cycles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    const int lb = m < 6 ? m : 6;
    uint64_t* lo_tab = reinterpret_cast<uint64_t*>(smem_raw + (sizeof(V) << m));
    uint64_t* hi_tab = lo_tab + (1 << lb);
    // offsets of tile-local index bits: low lb bits and the rest
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
    const uint32_t size = 1u << m;
    const uint32_t lmask = (1u << lb) - 1;
    for (uint64_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint64_t st = t >> rest;
        uint64_t tid = t & ((uint64_t(1) << rest) - 1);
        // insert zeros at the tile qubits (ascending)
        for (int b = 0; b < m; b++) {
            uint64_t low = (uint64_t(1) << tq.q[b]) - 1;
            tid = (tid & low) | ((tid & ~low) << 1);
        }
        V* __restrict__ g = s + ((st << n) | tid);
        constexpr int U = 4;
        for (uint32_t e0 = threadIdx.x; e0 < size; e0 += blockDim.x * U) {
            V r[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                uint32_t e = e0 + u * blockDim.x;
                if (e < size) r[u] = g[lo_tab[e & lmask] | hi_tab[e >> lb]];
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                uint32_t e = e0 + u * blockDim.x;
                if (e < size) tile[e] = r[u];
            }
        }
        __syncthreads();
        long long t0 = TIMED ? clock64() : 0;
        for (int i = 0; i < nops; i++) {
            tile_apply<V>(tile, ops[i], m, pool);
            __syncthreads();
            if (TIMED && threadIdx.x == 0) {
                long long t1 = clock64();
                atomicAdd(cycles + i, (unsigned long long)(t1 - t0));
                t0 = t1;
            }
        }
        for (uint32_t e = threadIdx.x; e < size; e += blockDim.x) g[lo_tab[e & lmask] | hi_tab[e >> lb]] = tile[e];
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

template <typename V, bool TIMED>
void tile_pass_t(const Batch& b, int m, const TileOp* ops, int nops, const double2* pool, const TilePass& hp,
                 unsigned long long* cycles) {
    TileQubits tq{};
    tq.m = m;
    for (int i = 0; i < m; i++) tq.q[i] = hp.qubits[i];
    const size_t smem = tile_smem_bytes(m, sizeof(V) == 8);
    static size_t configured[2][2] = {{0, 0}, {0, 0}};
    size_t& conf = configured[sizeof(V) == 8 ? 1 : 0][TIMED ? 1 : 0];
    if (smem > conf) {
        cudaFuncSetAttribute(k_tile<V, TIMED>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        // Largest carveout, so the occupancy below is what the launch gets.
        cudaFuncSetAttribute(k_tile<V, TIMED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             int(cudaSharedmemCarveoutMaxShared));
        conf = smem;
    }
    const uint64_t total = b.W << (b.n - m);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<V, TIMED>, kTileThreads, smem);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = std::min<uint64_t>(total, uint64_t(sm_count()) * per_sm);
    k_tile<V, TIMED><<<unsigned(grid), kTileThreads, smem, b.stream>>>(static_cast<V*>(b.amps), b.n, m, tq, ops, nops,
                                                                        pool, total, cycles);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(kCudaError, std::string("tile pass: ") + cudaGetErrorString(e));
}

}  // namespace

size_t tile_smem_bytes(int m, bool c64) {
    int lb = m < 6 ? m : 6;
    return (size_t(c64 ? 8 : 16) << m) + 8 * ((size_t(1) << lb) + (size_t(1) << (m - lb)));
}

void tile_pass(const Batch& b, const int* /*tile_qubits_dev*/, int m, const TileOp* ops_dev, int nops,
               const double2* pool_dev, const TilePass& host_pass, unsigned long long* cycles) {
    if (b.c64) {
        if (cycles)
            tile_pass_t<float2, true>(b, m, ops_dev, nops, pool_dev, host_pass, cycles);
        else
            tile_pass_t<float2, false>(b, m, ops_dev, nops, pool_dev, host_pass, nullptr);
    } else {
        if (cycles)
            tile_pass_t<double2, true>(b, m, ops_dev, nops, pool_dev, host_pass, cycles);
        else
            tile_pass_t<double2, false>(b, m, ops_dev, nops, pool_dev, host_pass, nullptr);
    }
}

}  // namespace k
}  // namespace dq

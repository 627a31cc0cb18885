// Shared-memory tile passes: many operations per HBM pass.
//
// A pass fixes a set T of m "tile qubits".  The state splits into 2^(n-m)
// tiles (all amplitudes that agree on the other qubits); a CTA loads one tile
// into shared memory, applies every operation of the pass (all of them act
// on qubits inside T, renumbered to tile-local bits), and writes the tile
// back.  Consecutive tile ids differ in the lowest qubits outside T, so CTAs
// that run together touch neighbouring sectors and L2 merges partial sectors
// when T does not start at qubit 0.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "compile.hpp"
#include "kernels.hpp"

namespace dq {

// Tile-local operation (all positions are tile-local bit indices).
struct TileOp {
    enum : int { kOne = 0, kX = 1, kDiagEntry = 2, kDiagFull = 3, kSwap = 4, kDense = 5 };
    int type;
    int k;                // qubits of a diagonal / dense matrix
    int nins;             // positions inserted when enumerating work items
    int ins[7];           // ascending
    int q[5];             // matrix qubits, q[0] = MSB of the matrix index
    uint32_t fixed;       // OR-ed after insertion (control values, diagonal pattern)
    uint32_t tbit;        // kOne / kX: target bit
    uint32_t lowbit, highbit;  // kSwap
    int mat;              // offset into the pass's double2 matrix pool
    int ngates;           // operations fused into this one
    uint32_t offs[32];    // kDense: offset of matrix index j
};

class CostModel;

struct TilePass {
    std::vector<int> qubits;  // ascending global positions of the m tile qubits
    std::vector<TileOp> ops;
    int op_begin = 0;         // index into the device op array
    // Register phases of the pass (phased.hpp): its block (index into the
    // executor's blocks, and first word in their device copy) and phase count;
    // nphases 0 when the pass runs one operation per sweep.
    int phase_block = -1, phase_begin = 0, nphases = 0;
    int raw_ops = 0;          // unfused operations covered (for statistics)
    std::vector<Operation> raw;  // filled when TilePlanOptions::keep_raw
    std::vector<size_t> op_index;  // the pass's operations: indices into the planned list, ascending
};

struct TilePlanOptions {
    int m = 12;          // tile qubits (2^m amplitudes in shared memory)
    int fuse = 2;        // widest fused dense operation
    int seeds = 6;       // candidate starts per pass
    bool c64 = false;
    // With a trained cost model, each pass takes the fusion width (1..3)
    // whose lowered operations have the smallest predicted cost.
    const CostModel* model = nullptr;
    std::vector<int>* chosen_widths = nullptr;  // filled per pass when given
    // Keep each pass's raw operations (for fused tensor-core blocks) instead
    // of lowering them to tile-local operations.
    bool keep_raw = false;
    // Qubits 0..pinned_low-1 belong to every tile, so each thread's run of
    // amplitudes in HBM is 2^pinned_low elements long (whole 32-byte sectors).
    int pinned_low = 0;
    // Partial plans kept by the pass search (1: the single best pass each
    // time).  Circuits of more than kPlanBeamMaxOps operations use 1.
    int beam = 1;
    // Tile qubits at or above spread_bit scatter the contiguous runs that the
    // tiles in flight together read (tiles in flight differ in the lowest
    // inflight_bits qubits outside the tile); a pass's spread, in quarters
    // (4 per tile qubit from spread_bit + 4 up, 3 per tile qubit in
    // [spread_bit, spread_bit + 4), less 12 per tile qubit that lengthens
    // those runs), is at most max_spread (-1: no limit).  See kFusedSpreadBit.
    int spread_bit = 0;
    int max_spread = -1;
    int inflight_bits = 9;
    // Shared-memory pass depth: at most this many operations per pass (0: no
    // limit).  Shallower passes cost more passes but less work per tile item.
    int max_pass_ops = 0;
};

constexpr size_t kPlanBeamMaxOps = 50000;
// Beam width of the prepared and per-call simulator plans (batched circuits
// plan with 1: hundreds of circuits are planned per call).
constexpr int kPlanBeam = 8;

// Widest dense operation a tile pass applies on CUDA cores (register budget).
constexpr int kTileMaxDense = 3;

// True for operations a tile pass can apply: unitary, unconditioned, and no
// dense matrix wider than kTileMaxDense qubits.
inline bool tileable(const Operation& op) {
    return op.is_unitary() && !(op.type == Operation::Dense && op.qubits.size() > size_t(kTileMaxDense));
}

// Plans passes over ops[begin, end) (tileable operations only).  Each pass is
// grown from one of the first `seeds` ready operations by one of two rules
// (add the ready operation needing the fewest new qubits; add the one whose new
// qubits let the most operations in per qubit), a beam of `beam` partial plans
// ranked by the operations covered keeps the best extensions, and the first
// plan to cover the range wins.  A pass lists its operations in circuit order.
std::vector<TilePass> plan_tiles(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                                 const TilePlanOptions& opt, std::vector<double2>* pool);

// Greedy dependency-respecting fusion of a topologically ordered op list into
// dense operations of at most `width` qubits (width 1 leaves gates alone).
std::vector<Operation> fuse_ops(const std::vector<Operation>& ops, int width);
// The same with a choice per block: of the qubit sets made from the block's
// first operation and up to `width` of the next few qubits, the set that
// absorbs the most operations (used for the 5-qubit tensor-core blocks, where
// every block costs the same whatever it holds).
std::vector<Operation> fuse_ops_lookahead(const std::vector<Operation>& ops, int width);

// ---------------------------------------------------------------------------
// Tensor-core fused blocks (complex64): a pass of 12 tile qubits whose
// operations are fused into 32x32 complex blocks, each applied as one
// 128 x 64 x 192 FP16 contraction (three products of f16 hi/lo parts, FP32
// accumulation, tiles scaled by a power of two) on tcgen05.
// ---------------------------------------------------------------------------
constexpr int kFusedM = 12;            // tile qubits of a fused pass
constexpr int kFusedPinned = 2;        // low qubits in every fused tile (32-byte runs of complex64)
// Fused passes keep their spread (TilePlanOptions) at most kFusedMaxSpread
// quarters over qubits from kFusedSpreadBit (2^20 complex64 = 8 MiB) up; about
// 2^9 tiles (148 CTAs x 4) are in flight.  Fitted to 450 single passes of three
// blocks over 327 tile qubit sets at 30 and 32 qubits: spread <= 24 took
// 0.95-1.17 of the median time, 25-28 1.29-1.44, above 28 1.29-1.76 (at 30
// qubits the median is 11.4 ms; five sets fall on the wrong side of 24).
constexpr int kFusedSpreadBit = 20;
constexpr int kFusedMaxSpread = 24;
constexpr int kFusedCols = 1 << (kFusedM - 5);
constexpr int kFusedUHalves = 2 * 64 * 64;  // U_hi and U_lo images of one block (f16)

// Byte offset in a block's tile operand (f16, K-major, 128-byte swizzled; K
// element 2*basis + re/im) of packed position (column << 5) | basis.  Linear
// over GF(2).
uint32_t fused_operand_offset(uint32_t packed);

// Device descriptor of one block.  An output at (column, basis) of this block
// goes to byte offset next_c[column] ^ next_b[basis]: in the next block's tile
// operand, or after the last block in the swizzled natural-order stage.
struct alignas(16) FusedBlock {
    uint32_t u_off;          // f16 offset of the block's U_hi/U_lo image in the pool
    uint32_t last;           // 1: outputs go to the stage
    uint32_t pad[2];
    uint16_t next_b[32];     // output basis -> destination offset part
    uint16_t next_c[128];    // output column -> destination offset part
};

struct FusedPass {
    std::vector<int> qubits;   // 12 ascending global positions
    int first_block = 0, nblocks = 0;
    uint16_t in_lo[64], in_hi[64];    // natural local index l -> operand offset of block 0 (lo ^ hi)
    uint16_t out_lo[64], out_hi[64];  // natural local index l -> stage offset (lo ^ hi)
    // The split of a loaded tile into block 0's operand: thread gt of a group
    // takes the amplitude pairs e = P(gt) | split_q[k], k = 0..15, where P
    // deposits bit b of 2*gt (b = 1..7) at local bit split_pos[b]; split_qoff[k]
    // is the operand offset of split_q[k].  Local bits 1..3 follow lane bits
    // 0..2 (16-byte reads of a quarter-warp stay in one 128-byte row); lane
    // bits 3 and 4 take the two local bits that give the warp's 4-byte stores
    // 32 distinct banks in block 0's layout, where two such bits exist.
    uint8_t split_pos[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    uint16_t split_q[16] = {};
    uint16_t split_qoff[16] = {};
    int raw_ops = 0;
    std::vector<int> block_gates;        // gates fused into each block
    std::vector<uint32_t> block_masks;   // each block's local qubits
};

// TMA loads of a fused pass's tiles.  The state buffer (8-byte complex64
// elements) is viewed as a tensor of up to 5 dimensions: dimension i covers
// global bits [lo[i], lo[i] + bits[i]) and the last dimension in use runs to
// the top of the buffer.  A tile is a box of that tensor: runs of tile qubits
// (chunks of at most 8 bits) are copied whole, the gaps between them one
// element at a time.  Tile qubits above the box come from `copies` boxes,
// copy c landing copy_bytes * c into the tile and starting copy_step[c]
// further along the last dimension; each box holds natural local order.
struct FusedTma {
    int ok = 0;          // 0: per-thread copies instead (shape or size outside the rules)
    int dims = 0;        // dimensions in use; the rest have extent 1
    int lo[5] = {0, 0, 0, 0, 0};
    int bits[5] = {0, 0, 0, 0, 0};  // span of a bounded dimension; the last one: its box bits
    uint32_t box[5] = {1, 1, 1, 1, 1};
    uint64_t extent[5] = {1, 1, 1, 1, 1};
    int copies = 1;
    uint32_t copy_bytes = 0;
    int32_t copy_step[16] = {};
};

// The TMA view for tiles of `tile_qubits` over `states` states of n qubits.
FusedTma fused_tma_plan(const std::vector<int>& tile_qubits, int n, uint64_t states);

// A pass's raw operations fused to `width` and lowered to tile-local
// operations for the CUDA-core tile kernel (matrices appended to `pool`).
void lower_pass_ops(const std::vector<Operation>& raw, const std::vector<int>& tile_qubits, int n, int width,
                    std::vector<double2>& pool, std::vector<TileOp>& out);

// Fuses a pass's operations into 5-qubit blocks and appends their descriptors
// and f16 hi/lo gate images (K-major, 128-byte swizzled operand layout).
FusedPass build_fused_pass(const std::vector<Operation>& pass_ops, const std::vector<int>& tile_qubits,
                           std::vector<FusedBlock>& blocks, std::vector<uint16_t>& upool);

// A fused pass with its own block descriptors and gate images (block offsets
// relative to its own arrays).
struct BuiltFusedPass {
    TilePass src;
    FusedPass fp;
    std::vector<FusedBlock> blocks;
    std::vector<uint16_t> upool;
};

// A pass's fixed cost (loads, stores, norms) in units of one block's: at 30
// qubits a pass of b blocks took about 3 + b ms (1 block 3.96 ms, 5 blocks
// 8.2-8.3 ms, 7 blocks 9.6-9.96 ms).
constexpr double kFusedPassCostBlocks = 3.0;
// The added cost of a pass whose spread exceeds kFusedMaxSpread by at most 4
// quarters, and by more (at 30 qubits about +4 ms and +8 ms).
constexpr double kFusedSpreadCostBlocks[2] = {4.0, 8.0};

// The candidate fused plans of ops[begin, end): one per spread cap (-1: no
// cap), each planned with kFusedM tile qubits, kFusedPinned pinned and beam
// kPlanBeam.  The plans share passes (same tile qubits, same operations), so
// each distinct pass is fused into blocks once.  `rule_cost` prices each plan
// by the hand-fitted rule: kFusedPassCostBlocks * passes + blocks +
// kFusedSpreadCostBlocks per pass over kFusedMaxSpread; `rule_choice` is the
// cheapest (the first on ties).
struct FusedPortfolio {
    int n = 0;
    std::vector<int> caps;
    std::vector<std::vector<TilePass>> plans;  // per cap: its passes (raw operations kept)
    std::vector<std::vector<size_t>> slots;    // per cap: each pass's index in `built`
    std::vector<BuiltFusedPass> built;         // distinct passes (their src left empty)
    std::vector<double> rule_cost;
    size_t rule_choice = 0;
};

// Spread caps of the portfolio.  The default set: kFusedMaxSpread and, where
// it can bind (every qubit from kFusedSpreadBit up in the tile exceeds it),
// also no cap and a cap 4 quarters lower.  The wide set, planned when a
// learned pass-cost model chooses among the plans, adds caps from 8 quarters
// below to 8 above.
std::vector<int> fused_caps(int n, bool wide);
FusedPortfolio fused_portfolio(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                               const TilePlanOptions& base, const std::vector<int>& caps);
// The passes of plan i (each with its source pass), moved out of the portfolio.
std::vector<BuiltFusedPass> take_fused_plan(FusedPortfolio& pf, size_t i);

// Plans ops[begin, end) as fused passes: the default portfolio's rule choice
// (the pass search follows ops covered, not blocks, so the caps give
// different plans).  `base` supplies seeds; the other planning fields are set
// here.
std::vector<BuiltFusedPass> plan_fused(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                                       const TilePlanOptions& base);

namespace k {
// One fused pass over every tile of every state (complex64 only).  err: device
// flag set to 3 when a bounded wait on an mbarrier runs out.
// in_norm (nullable): the previous fused pass's partial norm sums
// (fused_state_norm's output), divided out on load; tile_norm (W * 2^(n-12)
// doubles) receives each output tile's FP64 squared norm.  basis: every state
// is |0...0> on entry; the pass builds its input tiles itself and reads
// nothing of the state (which may hold anything).
void fused_pass(const Batch& b, const FusedPass& p, const FusedBlock* blocks_dev, const uint16_t* upool_dev,
                int* err_dev, const double* in_norm, double* tile_norm, bool basis = false);
// Partial sums of each state's tile norms, fused_norm_parts(n) per state in
// a fixed order (state st's norm is the in-order sum of norm[st*parts ..]).
int fused_norm_parts(int n);
void fused_state_norm(const Batch& b, const double* tile_norm, double* norm);
// Divides every state by the square root of its norm, summed from the partial
// sums fused_state_norm left (FP64 scale).
void fused_renormalize(const Batch& b, const double* norm);
size_t fused_smem_bytes();
// Sets the fused kernel's shared-memory attributes on the current device (once).
void fused_configure();
// Failure-path tests: gate images of fused steps >= withhold_step are never
// fetched, and every bounded wait of the fused kernel gives up after wait_ms
// (<= 0: the default of about 2 s).  ~0 restores normal operation.
void set_fused_fault(uint64_t withhold_step, double wait_ms);
}  // namespace k

namespace k {
// One pass over every tile of every state in the batch.  With `cycles`, thread
// 0 of each CTA adds the clock64() cycles every operation took on each tile it
// processed (one slot per operation), for the cost model's training data.
void tile_pass(const Batch& b, const int* tile_qubits_dev, int m, const TileOp* ops_dev, int nops,
               const double2* pool_dev, const TilePass& host_pass, unsigned long long* cycles = nullptr);
size_t tile_smem_bytes(int m, bool c64);
}  // namespace k

}  // namespace dq

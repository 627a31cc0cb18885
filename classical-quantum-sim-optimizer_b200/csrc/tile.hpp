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
    int raw_ops = 0;          // unfused operations covered (for statistics)
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
};

// Widest dense operation a tile pass applies on CUDA cores (register budget).
constexpr int kTileMaxDense = 3;

// True for operations a tile pass can apply: unitary, unconditioned, and no
// dense matrix wider than kTileMaxDense qubits.
inline bool tileable(const Operation& op) {
    return op.is_unitary() && !(op.type == Operation::Dense && op.qubits.size() > size_t(kTileMaxDense));
}

// Plans passes over ops[begin, end) (tileable operations only).
std::vector<TilePass> plan_tiles(const std::vector<Operation>& ops, size_t begin, size_t end, int n,
                                 const TilePlanOptions& opt, std::vector<double2>* pool);

// Greedy dependency-respecting fusion of a topologically ordered op list into
// dense operations of at most `width` qubits (width 1 leaves gates alone).
std::vector<Operation> fuse_ops(const std::vector<Operation>& ops, int width);

namespace k {
// One pass over every tile of every state in the batch.  With `cycles`, thread
// 0 of each CTA adds the clock64() cycles every operation took on each tile it
// processed (one slot per operation), for the cost model's training data.
void tile_pass(const Batch& b, const int* tile_qubits_dev, int m, const TileOp* ops_dev, int nops,
               const double2* pool_dev, const TilePass& host_pass, unsigned long long* cycles = nullptr);
size_t tile_smem_bytes(int m, bool c64);
}  // namespace k

}  // namespace dq

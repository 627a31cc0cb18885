// Tile passes in register phases (phased.cu).
//
// A tile pass holds 2^m amplitudes in shared memory and applies its fused
// operations one after another.  Applied one per sweep, every operation reads
// and writes the whole tile in shared memory (32 bytes per amplitude for
// complex128), and that traffic, not FP64 arithmetic, bounds the sweep.  Here
// the pass's operations are grouped into phases.  A phase names three tile
// qubits, the register qubits: each thread loads the 8 amplitudes that differ
// only in them into registers, applies every operation of the phase there and
// stores them back.  Shared memory is then read and written once per phase
// instead of once per operation.  Four register qubits take about twice the
// operations per phase on brickwork passes, but 16 complex128 amplitudes per
// thread leave room for one CTA per SM only, and measured slower.
//
// An operation joins a phase when its targets (the qubits whose amplitudes it
// mixes) are among the phase's register qubits and it commutes with every
// earlier operation of the pass still waiting for a later phase.  Diagonal
// operations have no targets; controls and diagonal patterns are read off
// each amplitude's tile index.  Within a phase the operations keep their
// pass order.
//
// A pass's phases, operations and matrices form one block of 16-byte words.
// A block that fits the kernel-parameter space travels as a launch argument:
// every thread reads the same word at the same time, which the constant cache
// serves without the load/store pipe the amplitudes need.  Larger blocks are
// read from device memory.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "kernels.hpp"
#include "tile.hpp"

namespace dq {

#ifndef DQ_PHASE_REG_BITS
#define DQ_PHASE_REG_BITS 3
#endif
constexpr int kPhaseRegBits = DQ_PHASE_REG_BITS;  // register qubits per phase (3 or 4)
static_assert(kPhaseRegBits == 3 || kPhaseRegBits == 4, "three or four register qubits");
constexpr int kPhaseEntries = 1 << kPhaseRegBits;  // amplitudes per thread and slot
constexpr int kPhaseMaxSlotBits = 16;

// Block layout (uint4 words, indices relative to the block):
//   phase p at 6p: w0 = {first op word, op count, slot bits, 0};
//     w1 = register qubit i as (1 << q) | (swizzled (1 << q)) << 16, i < 4;
//     w2..w5 = slot bit i likewise, i < 16;
//   operation at 2 words: {code, first matrix word, condition mask, value},
//     {k, diagonal qubits 0-3 and 4-7 as bytes, 0};
//   matrices: one double2 per word.
constexpr int kPhaseWords = 6;
constexpr int kPhaseOpWords = 2;
constexpr int kPhaseParamWords = 2040;  // largest block passed as a kernel argument (32,640 bytes)

// Operation codes: 0-3 one-qubit matrix on register qubit 0-3; 4-7 X; 8-13
// two-qubit dense on register qubits (1,0), (2,0), (2,1), (3,0), (3,1), (3,2)
// (matrix index bit 1 on the higher one); 14-17 three-qubit dense on (2,1,0),
// (3,1,0), (3,2,0), (3,2,1) (matrix index bit 2 on the highest); 18-23 swap of
// the pairs in the two-qubit order; 24 one diagonal entry; 25 a full diagonal
// over k tile qubits (the first the MSB of the table index).  Operations with
// a condition act where (tile index & mask) == value.
enum PhaseCode : int { kPhOne = 0, kPhX = 4, kPhD2 = 8, kPhD3 = 14, kPhSwap = 18, kPhDiagEntry = 24, kPhDiagFull = 25 };

// Index of register-qubit pair (h > l) in the two-qubit order above, and of
// triple (a > b > c) in the three-qubit order.
__host__ __device__ constexpr int phase_pair(int h, int l) { return h * (h - 1) / 2 + l; }
__host__ __device__ constexpr int phase_triple(int a, int b, int c) { return a == 2 ? 0 : b == 1 ? 1 : c == 0 ? 2 : 3; }

// The swizzle of tile index e: its low g bits XOR the XOR of every higher
// g-bit chunk (g = 3 for complex128, 4 for complex64), so the 2^g lanes whose
// slot bits come from g tile qubits of distinct residues mod g hit distinct
// bank groups.
inline uint32_t phase_swizzle(uint32_t e, int g) {
    uint32_t f = 0;
    for (uint32_t x = e >> g; x; x >>= g) f ^= x;
    return e ^ (f & ((1u << g) - 1));
}

// True when a pass of m tile qubits can run in phases.
inline bool phase_supported(int m) { return m >= kPhaseRegBits + 2 && m - kPhaseRegBits <= kPhaseMaxSlotBits; }

// Groups `ops` (one pass, m tile qubits, matrices in `pool`) into phases and
// writes the pass's block.  Returns the number of phases.
int plan_phases(const std::vector<TileOp>& ops, int m, bool c64, const std::vector<double2>& pool,
                std::vector<uint4>& block);

namespace k {

// One tile pass in phases.  `block` is the host copy of the pass's block and
// `block_dev` the same words on the device (read when the block is larger
// than the kernel-parameter space).
void tile_pass_phased(const Batch& b, const TilePass& host_pass, int nphases, const std::vector<uint4>& block,
                      const uint4* block_dev);

}  // namespace k
}  // namespace dq

// Gate tables and the Operation lowering with single-qubit fusion.
//
// Gate matrices follow src/gates.rs:23-274 and gate_matrix_1q in
// src/types.rs:303-344 (FP64, libm cos/sin, num-complex arithmetic).  The
// lowering follows src/monolithic/statevector/execution.rs:21-416: X and
// diagonal detection, per-qubit fusion of 1q gates flushed by a touching
// multi-qubit operation, and a full flush at Measure and Barrier.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "common.hpp"

namespace dq {

struct Control {
    uint64_t qubit;
    bool value;
};

struct Operation {
    // Noop appears only as the operation of a Conditional (a conditioned
    // barrier), which the reference keeps in the plan (execution.rs:246-250, 406-409).
    enum Type { One, X, Swap, Diagonal, Dense, Measure, Reset, Conditional, Noop };
    Type type = One;
    uint64_t target = 0;           // One, X
    uint64_t a = 0, b = 0;         // Swap
    Mat2 m{};                      // One
    std::vector<Control> controls; // One, X, Swap
    std::vector<uint64_t> qubits;  // Diagonal, Dense (qubits[0] = MSB of the matrix index)
    std::vector<cplx> values;      // Diagonal: 2^k entries; Dense: row-major 2^k x 2^k
    uint64_t qubit = 0, cbit = 0;  // Measure, Reset
    Condition condition;           // Conditional
    std::shared_ptr<Operation> inner;
    int fused_count = 1;           // operations multiplied into this one by a fusion pass

    bool is_unitary() const { return type != Measure && type != Reset && type != Conditional; }
    // Qubits the operation reads or writes (conditions excluded).
    std::vector<uint64_t> touched() const;
};

// Returns the 1q matrix of a single-qubit instruction, or false.
bool gate_matrix_1q(const Instruction& in, uint64_t* qubit, Mat2* m);

// Operation::compile for one instruction (no fusion); throws Error(kValueError).
// Returns false for a no-op (Barrier, remote_barrier).
bool compile_instruction(const Instruction& in, Operation* out);

// compile: instructions -> fused operation list.
std::vector<Operation> compile(const std::vector<Instruction>& instructions);

// Deterministic JSON dump (hex bit patterns for doubles) used by host tests.
std::string dump_operations(const std::vector<Operation>& ops);

// Dense matrices of multi-qubit gates (row-major, qubits[0] = MSB).
std::vector<cplx> gate_matrix_dense(const std::string& which, double theta);

}  // namespace dq

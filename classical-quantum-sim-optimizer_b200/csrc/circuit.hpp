// Circuit transport IR, parsing and validation.
//
// Mirrors the serde schema of src/types.rs:7-296 (an internally tagged enum
// on "kind", 48 variants) and the rejection rules of src/validation.rs:5-182
// plus src/monolithic/statevector/validation.rs:3-12.
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "common.hpp"

namespace dq {

enum class Kind {
    Id, X, Y, Z, H, S, Sdg, T, Tdg, Sx, Sxdg,
    U3, U2, U1, U, P, Rx, Ry, Rz, U0,
    Cx, Cz, Cy, Ch, Swap, Csx,
    Crx, Cry, Crz, Cu1, Cp, Cu3, Cu, Rxx, Rzz,
    Ccx, Cswap, Rccx, Rc3x, C3x, C3sqrtx, C4x,
    Gate, Measure, Reset, Conditional, Barrier, Classical,
};

struct Condition {
    uint64_t creg_base = 0, creg_size = 0, creg_value = 0;
};

// Parameter slots: theta, phi, lam, gamma.
enum Param { kTheta = 0, kPhi = 1, kLam = 2, kGamma = 3 };

struct Instruction {
    Kind kind = Kind::Barrier;
    std::vector<uint64_t> qubits;  // operands in Instruction::qubits order (types.rs:346-463)
    double p[4] = {0, 0, 0, 0};
    uint64_t cbit = 0;
    std::string name;             // Gate / Classical
    std::vector<double> params;   // Gate
    Condition condition;          // Conditional
    std::shared_ptr<Instruction> op;  // Conditional

    // Instruction::qubits, with Conditional forwarding to its operation.
    const std::vector<uint64_t>& operands() const { return kind == Kind::Conditional ? op->operands() : qubits; }
};

struct Register {
    std::string name;
    uint64_t size = 0, base = 0;
};

struct Circuit {
    std::vector<std::pair<std::string, Register>> qregs, cregs;
    std::vector<Instruction> instructions;
    uint64_t num_qubits() const;  // Circuit::num_qubits, types.rs:24-30
    uint64_t num_cbits() const;
};

// serde_json::from_str::<Circuit>; throws Error(kValueError, "Circuit JSON parse error: ...").
Circuit parse_circuit(const char* text, size_t len);

// validate_circuit (statevector flavour); throws Error(kValueError, ...).
void validate_circuit(const Circuit& c);

// Instruction name as it appears in the "kind" tag.
const char* kind_name(Kind k);

}  // namespace dq

#include "circuit.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>

#include "json.hpp"

namespace dq {
namespace {

// One entry per Instruction variant: the "kind" tag, the operand fields in
// Instruction::qubits order, and the f64 fields with their parameter slots.
struct Spec {
    const char* tag;
    Kind kind;
    std::vector<const char*> operands;
    std::vector<std::pair<const char*, int>> params;
};

const std::vector<Spec>& specs() {
    static const std::vector<Spec> table = {
        {"id", Kind::Id, {"qubit"}, {}},
        {"x", Kind::X, {"qubit"}, {}},
        {"y", Kind::Y, {"qubit"}, {}},
        {"z", Kind::Z, {"qubit"}, {}},
        {"h", Kind::H, {"qubit"}, {}},
        {"s", Kind::S, {"qubit"}, {}},
        {"sdg", Kind::Sdg, {"qubit"}, {}},
        {"t", Kind::T, {"qubit"}, {}},
        {"tdg", Kind::Tdg, {"qubit"}, {}},
        {"sx", Kind::Sx, {"qubit"}, {}},
        {"sxdg", Kind::Sxdg, {"qubit"}, {}},
        {"u3", Kind::U3, {"qubit"}, {{"theta", kTheta}, {"phi", kPhi}, {"lam", kLam}}},
        {"u2", Kind::U2, {"qubit"}, {{"phi", kPhi}, {"lam", kLam}}},
        {"u1", Kind::U1, {"qubit"}, {{"lam", kLam}}},
        {"u", Kind::U, {"qubit"}, {{"theta", kTheta}, {"phi", kPhi}, {"lam", kLam}}},
        {"p", Kind::P, {"qubit"}, {{"lam", kLam}}},
        {"rx", Kind::Rx, {"qubit"}, {{"theta", kTheta}}},
        {"ry", Kind::Ry, {"qubit"}, {{"theta", kTheta}}},
        {"rz", Kind::Rz, {"qubit"}, {{"phi", kPhi}}},
        {"u0", Kind::U0, {"qubit"}, {}},
        {"cx", Kind::Cx, {"control", "target"}, {}},
        {"cz", Kind::Cz, {"control", "target"}, {}},
        {"cy", Kind::Cy, {"control", "target"}, {}},
        {"ch", Kind::Ch, {"control", "target"}, {}},
        {"swap", Kind::Swap, {"a", "b"}, {}},
        {"csx", Kind::Csx, {"control", "target"}, {}},
        {"crx", Kind::Crx, {"control", "target"}, {{"theta", kTheta}}},
        {"cry", Kind::Cry, {"control", "target"}, {{"theta", kTheta}}},
        {"crz", Kind::Crz, {"control", "target"}, {{"lam", kLam}}},
        {"cu1", Kind::Cu1, {"control", "target"}, {{"lam", kLam}}},
        {"cp", Kind::Cp, {"control", "target"}, {{"lam", kLam}}},
        {"cu3", Kind::Cu3, {"control", "target"}, {{"theta", kTheta}, {"phi", kPhi}, {"lam", kLam}}},
        {"cu", Kind::Cu, {"control", "target"}, {{"theta", kTheta}, {"phi", kPhi}, {"lam", kLam}, {"gamma", kGamma}}},
        {"rxx", Kind::Rxx, {"a", "b"}, {{"theta", kTheta}}},
        {"rzz", Kind::Rzz, {"a", "b"}, {{"theta", kTheta}}},
        {"ccx", Kind::Ccx, {"control1", "control2", "target"}, {}},
        {"cswap", Kind::Cswap, {"control", "target1", "target2"}, {}},
        {"rccx", Kind::Rccx, {"control1", "control2", "target"}, {}},
        {"rc3x", Kind::Rc3x, {"control1", "control2", "control3", "target"}, {}},
        {"c3x", Kind::C3x, {"control1", "control2", "control3", "target"}, {}},
        {"c3sqrtx", Kind::C3sqrtx, {"control1", "control2", "control3", "target"}, {}},
        {"c4x", Kind::C4x, {"control1", "control2", "control3", "control4", "target"}, {}},
        {"gate", Kind::Gate, {}, {}},
        {"measure", Kind::Measure, {"qubit"}, {}},
        {"reset", Kind::Reset, {"qubit"}, {}},
        {"conditional", Kind::Conditional, {}, {}},
        {"barrier", Kind::Barrier, {}, {}},
        {"classical", Kind::Classical, {}, {}},
    };
    return table;
}

[[noreturn]] void parse_fail(const std::string& msg) { fail(kValueError, "Circuit JSON parse error: " + msg); }

const json::Value& field(const json::Value& obj, const char* key) {
    int c = obj.count(key);
    if (c == 0) parse_fail(std::string("missing field `") + key + "`");
    if (c > 1) parse_fail(std::string("duplicate field `") + key + "`");
    return *obj.find(key);
}

uint64_t as_usize(const json::Value& v, const char* what) {
    if (v.type != json::Type::Int || v.negative || v.int_overflow)
        parse_fail(std::string("invalid type or value for `") + what + "`, expected usize");
    return v.u;
}

double as_f64(const json::Value& v, const char* what) {
    if (v.type != json::Type::Int && v.type != json::Type::Float)
        parse_fail(std::string("invalid type for `") + what + "`, expected f64");
    return v.f;
}

const std::string& as_string(const json::Value& v, const char* what) {
    if (v.type != json::Type::String) parse_fail(std::string("invalid type for `") + what + "`, expected a string");
    return v.s;
}

Instruction parse_instruction(const json::Value& v) {
    if (v.type != json::Type::Object) parse_fail("expected an instruction object");
    const std::string& tag = as_string(field(v, "kind"), "kind");
    const Spec* spec = nullptr;
    for (auto& s : specs())
        if (tag == s.tag) spec = &s;
    if (!spec) parse_fail("unknown variant `" + tag + "`");
    Instruction in;
    in.kind = spec->kind;
    for (const char* f : spec->operands) in.qubits.push_back(as_usize(field(v, f), f));
    for (auto& pr : spec->params) in.p[pr.second] = as_f64(field(v, pr.first), pr.first);
    switch (in.kind) {
        case Kind::Measure: in.cbit = as_usize(field(v, "cbit"), "cbit"); break;
        case Kind::Gate: {
            in.name = as_string(field(v, "name"), "name");
            const json::Value& ps = field(v, "params");
            if (ps.type != json::Type::Array) parse_fail("invalid type for `params`, expected a sequence");
            for (auto& x : ps.arr) in.params.push_back(as_f64(x, "params"));
            const json::Value& qs = field(v, "qubits");
            if (qs.type != json::Type::Array) parse_fail("invalid type for `qubits`, expected a sequence");
            for (auto& x : qs.arr) in.qubits.push_back(as_usize(x, "qubits"));
            break;
        }
        case Kind::Classical: in.name = as_string(field(v, "name"), "name"); break;
        case Kind::Conditional: {
            const json::Value& c = field(v, "condition");
            if (c.type != json::Type::Object) parse_fail("invalid type for `condition`");
            in.condition.creg_base = as_usize(field(c, "creg_base"), "creg_base");
            in.condition.creg_size = as_usize(field(c, "creg_size"), "creg_size");
            in.condition.creg_value = as_usize(field(c, "creg_value"), "creg_value");
            in.op = std::make_shared<Instruction>(parse_instruction(field(v, "op")));
            break;
        }
        default: break;
    }
    return in;
}

std::vector<std::pair<std::string, Register>> parse_registers(const json::Value& v) {
    if (v.type != json::Type::Object) parse_fail("invalid type for registers, expected a map");
    std::vector<std::pair<std::string, Register>> out;
    for (auto& kv : v.obj) {
        const json::Value& r = kv.second;
        if (r.type != json::Type::Object) parse_fail("invalid type for a register");
        Register reg;
        reg.name = as_string(field(r, "name"), "name");
        reg.size = as_usize(field(r, "size"), "size");
        reg.base = as_usize(field(r, "base"), "base");
        // A HashMap keeps the last duplicate key.
        bool replaced = false;
        for (auto& e : out)
            if (e.first == kv.first) {
                e.second = reg;
                replaced = true;
            }
        if (!replaced) out.emplace_back(kv.first, reg);
    }
    return out;
}

using Ranges = std::vector<std::pair<uint64_t, uint64_t>>;

Ranges register_ranges(const std::vector<std::pair<std::string, Register>>& regs, const char* kind) {
    Ranges ranges;
    for (auto& kv : regs) {
        const Register& r = kv.second;
        if (r.base > kU64Max - r.size)
            fail(kValueError, std::string(kind) + " register \"" + kv.first + "\" has an overflowing range");
        if (r.size != 0) ranges.emplace_back(r.base, r.base + r.size);
    }
    std::sort(ranges.begin(), ranges.end());
    for (size_t i = 1; i < ranges.size(); i++)
        if (ranges[i].first < ranges[i - 1].second) fail(kValueError, std::string("Overlapping ") + kind + " registers");
    return ranges;
}

bool declared(uint64_t i, const Ranges& r) {
    for (auto& x : r)
        if (x.first <= i && i < x.second) return true;
    return false;
}

std::string lower(const std::string& s) {
    std::string o = s;
    for (auto& c : o) c = char(std::tolower(static_cast<unsigned char>(c)));
    return o;
}

struct GenericSpec {
    const char* name;
    int arity;  // -1: any
    size_t params;
};
const GenericSpec kGeneric[] = {
    {"remote_link_phi_plus", 2, 0}, {"remote_link_psi_minus", 2, 0}, {"remote_link_psi_plus", 2, 0},
    {"nonlocal_cz", 2, 0},          {"remote_cz", 2, 0},             {"remote_cx", 2, 0},
    {"remote_epr", 2, 0},           {"epr", 2, 0},                   {"remote_rzz", 2, 1},
    {"remote_cu1", 2, 1},           {"remote_barrier", -1, 0},
};

bool finite_all(std::initializer_list<double> xs) {
    for (double x : xs)
        if (!std::isfinite(x)) return false;
    return true;
}

// validate_instruction, src/validation.rs:44-182
void validate_instruction(const Instruction& in, const Ranges& qubits, const Ranges& cbits) {
    if (in.kind == Kind::Conditional) {
        const Condition& c = in.condition;
        if (c.creg_size == 0 || c.creg_size > 64) fail(kValueError, "Condition width must be between 1 and 64 bits");
        if (c.creg_base > kU64Max - c.creg_size) fail(kValueError, "Condition has an overflowing classical range");
        for (uint64_t bit = c.creg_base; bit < c.creg_base + c.creg_size; bit++)
            if (!declared(bit, cbits)) fail(kValueError, "Condition refers to undeclared classical bits");
        if (c.creg_size < 64 && c.creg_value >= (uint64_t(1) << c.creg_size))
            fail(kValueError, "Condition value does not fit its classical width");
        validate_instruction(*in.op, qubits, cbits);
        return;
    }
    const auto& ops = in.qubits;
    for (size_t i = 0; i < ops.size(); i++) {
        if (!declared(ops[i], qubits))
            fail(kValueError, "Qubit " + std::to_string(ops[i]) + " is not declared by a quantum register");
        for (size_t j = 0; j < i; j++)
            if (ops[j] == ops[i])
                fail(kValueError, "Gate operands must be distinct; qubit " + std::to_string(ops[i]) + " is repeated");
    }
    if (in.kind == Kind::Measure && !declared(in.cbit, cbits))
        fail(kValueError, "Classical bit " + std::to_string(in.cbit) + " is not declared by a classical register");
    if (in.kind == Kind::Classical) fail(kValueError, "Unsupported classical operation: \"" + in.name + "\"");
    if (in.kind == Kind::Gate) {
        std::string nm = lower(in.name);
        const GenericSpec* g = nullptr;
        for (auto& s : kGeneric)
            if (nm == s.name) g = &s;
        if (!g) fail(kValueError, "Unsupported generic gate: \"" + in.name + "\". Decompose it before simulating.");
        if (g->arity >= 0 && in.qubits.size() != size_t(g->arity))
            fail(kValueError, "Gate \"" + in.name + "\" requires " + std::to_string(g->arity) + " qubits, received " +
                                  std::to_string(in.qubits.size()));
        if (in.params.size() != g->params)
            fail(kValueError, "Gate \"" + in.name + "\" requires " + std::to_string(g->params) +
                                  " parameters, received " + std::to_string(in.params.size()));
    }
    bool fin = true;
    const double* p = in.p;
    switch (in.kind) {
        case Kind::U3: case Kind::U: case Kind::Cu3: fin = finite_all({p[kTheta], p[kPhi], p[kLam]}); break;
        case Kind::Cu: fin = finite_all({p[kTheta], p[kPhi], p[kLam], p[kGamma]}); break;
        case Kind::U2: fin = finite_all({p[kPhi], p[kLam]}); break;
        case Kind::U1: case Kind::P: case Kind::Crz: case Kind::Cu1: case Kind::Cp: fin = std::isfinite(p[kLam]); break;
        case Kind::Rx: case Kind::Ry: case Kind::Crx: case Kind::Cry: case Kind::Rxx: case Kind::Rzz:
            fin = std::isfinite(p[kTheta]);
            break;
        case Kind::Rz: fin = std::isfinite(p[kPhi]); break;
        case Kind::Gate:
            for (double x : in.params)
                if (!std::isfinite(x)) fin = false;
            break;
        default: break;
    }
    if (!fin) fail(kValueError, "Gate parameters must be finite numbers");
    switch (in.kind) {
        case Kind::U3: case Kind::U2: case Kind::U: case Kind::Cu3: case Kind::Cu:
            if (!std::isfinite(p[kPhi] + p[kLam])) fail(kValueError, "The combined phase phi + lam must be finite");
            break;
        default: break;
    }
}

}  // namespace

const char* kind_name(Kind k) {
    for (auto& s : specs())
        if (s.kind == k) return s.tag;
    return "?";
}

uint64_t Circuit::num_qubits() const {
    uint64_t m = 0;
    for (auto& kv : qregs) m = std::max(m, kv.second.base + kv.second.size);
    return m;
}

uint64_t Circuit::num_cbits() const {
    uint64_t m = 0;
    for (auto& kv : cregs) m = std::max(m, kv.second.base + kv.second.size);
    return m;
}

Circuit parse_circuit(const char* text, size_t len) {
    json::Value root;
    try {
        root = json::parse(text, len);
    } catch (const std::runtime_error& e) {
        parse_fail(e.what());
    }
    if (root.type != json::Type::Object) parse_fail("invalid type, expected struct Circuit");
    Circuit c;
    c.qregs = parse_registers(field(root, "qregs"));
    if (root.count("cregs") > 1) parse_fail("duplicate field `cregs`");
    if (const json::Value* cr = root.find("cregs")) c.cregs = parse_registers(*cr);
    const json::Value& insts = field(root, "instructions");
    if (insts.type != json::Type::Array) parse_fail("invalid type for `instructions`, expected a sequence");
    c.instructions.reserve(insts.arr.size());
    for (auto& v : insts.arr) c.instructions.push_back(parse_instruction(v));
    return c;
}

void validate_circuit(const Circuit& c) {
    Ranges qubits = register_ranges(c.qregs, "quantum");
    Ranges cbits = register_ranges(c.cregs, "classical");
    for (size_t i = 0; i < c.instructions.size(); i++) {
        try {
            validate_instruction(c.instructions[i], qubits, cbits);
        } catch (const Error& e) {
            fail(kValueError, "Instruction " + std::to_string(i) + ": " + e.what());
        }
    }
    if (c.num_qubits() >= 64) fail(kValueError, "Statevector qubit count must be less than 64");
}

}  // namespace dq

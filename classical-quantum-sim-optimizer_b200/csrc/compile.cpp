#include "compile.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>

namespace dq {
namespace {

constexpr double kS2 = 0.7071067811865476;  // FRAC_1_SQRT_2

Mat2 mat(cplx a, cplx b, cplx c, cplx d) {
    Mat2 m;
    m[0][0] = a;
    m[0][1] = b;
    m[1][0] = c;
    m[1][1] = d;
    return m;
}

const Mat2 kI = mat(cplx(1), cplx(0), cplx(0), cplx(1));
const Mat2 kX = mat(cplx(0), cplx(1), cplx(1), cplx(0));
const Mat2 kY = mat(cplx(0), cplx(0, -1), cplx(0, 1), cplx(0));
const Mat2 kZ = mat(cplx(1), cplx(0), cplx(0), cplx(-1));

Mat2 g_h() { return mat(cplx(kS2), cplx(kS2), cplx(kS2), cplx(-kS2)); }
Mat2 g_s() { return mat(cplx(1), cplx(0), cplx(0), cplx(0, 1)); }
Mat2 g_sdg() { return mat(cplx(1), cplx(0), cplx(0), cplx(0, -1)); }
Mat2 g_t() { return mat(cplx(1), cplx(0), cplx(0), cplx(kS2, kS2)); }
Mat2 g_tdg() { return mat(cplx(1), cplx(0), cplx(0), cplx(kS2, -kS2)); }
Mat2 g_sx() { return mat(cplx(0.5, 0.5), cplx(0.5, -0.5), cplx(0.5, -0.5), cplx(0.5, 0.5)); }
Mat2 g_sxdg() { return mat(cplx(0.5, -0.5), cplx(0.5, 0.5), cplx(0.5, 0.5), cplx(0.5, -0.5)); }

// gates.rs:65-74
Mat2 g_u3(double theta, double phi, double lam) {
    double ct = std::cos(theta / 2.0), st = std::sin(theta / 2.0);
    return mat(cplx(ct), -(cplx(std::cos(lam), std::sin(lam)) * cplx(st)), cplx(std::cos(phi), std::sin(phi)) * cplx(st),
               cplx(std::cos(phi + lam), std::sin(phi + lam)) * cplx(ct));
}
Mat2 g_u2(double phi, double lam) { return g_u3(M_PI / 2.0, phi, lam); }
Mat2 g_p(double lam) { return mat(cplx(1), cplx(0), cplx(0), cplx(std::cos(lam), std::sin(lam))); }
Mat2 g_rx(double t) {
    double c2 = std::cos(t / 2.0), s2 = std::sin(t / 2.0);
    return mat(cplx(c2), cplx(0, -s2), cplx(0, -s2), cplx(c2));
}
Mat2 g_ry(double t) {
    double c2 = std::cos(t / 2.0), s2 = std::sin(t / 2.0);
    return mat(cplx(c2), cplx(-s2), cplx(s2), cplx(c2));
}
Mat2 g_rz(double phi) {
    return mat(cplx(std::cos(-phi / 2.0), std::sin(-phi / 2.0)), cplx(0), cplx(0),
               cplx(std::cos(phi / 2.0), std::sin(phi / 2.0)));
}

std::vector<cplx> identity(int dim) {
    std::vector<cplx> m(size_t(dim) * dim, cplx(0));
    for (int i = 0; i < dim; i++) m[size_t(i) * dim + i] = cplx(1);
    return m;
}

// Operation::one, execution.rs:66-87
Operation op_one(uint64_t target, const Mat2& m, std::vector<Control> controls) {
    Operation op;
    if (m == kX) {
        op.type = Operation::X;
        op.target = target;
        op.controls = std::move(controls);
        return op;
    }
    if (m[0][1] == cplx(0) && m[1][0] == cplx(0)) {
        op.type = Operation::Diagonal;
        for (auto& c : controls) op.qubits.push_back(c.qubit);
        op.qubits.push_back(target);
        op.values.assign(size_t(1) << op.qubits.size(), cplx(1));
        size_t index = 0;
        for (auto& c : controls) index = (index << 1) | size_t(c.value);
        index <<= 1;
        op.values[index] = m[0][0];
        op.values[index + 1] = m[1][1];
        return op;
    }
    op.type = Operation::One;
    op.target = target;
    op.m = m;
    op.controls = std::move(controls);
    return op;
}

// Operation::dense, execution.rs:89-106
Operation op_dense(std::vector<uint64_t> qubits, const std::vector<cplx>& m) {
    size_t dim = size_t(1) << qubits.size();
    bool diag = true;
    for (size_t i = 0; i < dim && diag; i++)
        for (size_t j = 0; j < dim; j++)
            if (i != j && m[i * dim + j] != cplx(0)) {
                diag = false;
                break;
            }
    Operation op;
    op.qubits = std::move(qubits);
    if (diag) {
        op.type = Operation::Diagonal;
        for (size_t i = 0; i < dim; i++) op.values.push_back(m[i * dim + i]);
    } else {
        op.type = Operation::Dense;
        op.values = m;
    }
    return op;
}

Operation op_swap(uint64_t a, uint64_t b, std::vector<Control> controls) {
    Operation op;
    op.type = Operation::Swap;
    op.a = a;
    op.b = b;
    op.controls = std::move(controls);
    return op;
}

Operation op_x(uint64_t target, std::vector<Control> controls) {
    Operation op;
    op.type = Operation::X;
    op.target = target;
    op.controls = std::move(controls);
    return op;
}

std::string lower(const std::string& s) {
    std::string o = s;
    for (auto& c : o) c = char(std::tolower(static_cast<unsigned char>(c)));
    return o;
}

}  // namespace

std::vector<cplx> gate_matrix_dense(const std::string& which, double theta) {
    const cplx o(0);
    if (which == "rxx") {  // gates.rs:189-198
        double cv = std::cos(theta / 2.0), sv = std::sin(theta / 2.0);
        cplx c(cv), m(0, -sv);
        return {c, o, o, m, o, c, m, o, o, m, c, o, m, o, o, c};
    }
    if (which == "rzz") {  // gates.rs:199-204
        cplx ep(std::cos(theta / 2.0), std::sin(theta / 2.0));
        cplx em(std::cos(theta / 2.0), -std::sin(theta / 2.0));
        return {em, o, o, o, o, ep, o, o, o, o, ep, o, o, o, o, em};
    }
    if (which == "rccx") {  // gates.rs:210-219
        auto m = identity(8);
        m[5 * 8 + 5] = cplx(-1);
        m[6 * 8 + 6] = cplx(0);
        m[7 * 8 + 7] = cplx(0);
        m[6 * 8 + 7] = cplx(0, -1);
        m[7 * 8 + 6] = cplx(0, 1);
        return m;
    }
    if (which == "rc3x") {  // gates.rs:225-235
        auto m = identity(16);
        m[12 * 16 + 12] = cplx(0, 1);
        m[13 * 16 + 13] = cplx(0, -1);
        m[14 * 16 + 14] = cplx(0);
        m[15 * 16 + 15] = cplx(0);
        m[14 * 16 + 15] = cplx(1);
        m[15 * 16 + 14] = cplx(-1);
        return m;
    }
    const cplx s(kS2), ns(-kS2);
    if (which == "psi_minus") return {o, s, o, s, s, o, s, o, ns, o, s, o, o, ns, o, s};  // gates.rs:240-248
    if (which == "psi_plus") {  // gates.rs:250-262: rows 2 and 3 of psi_minus negated
        auto m = gate_matrix_dense("psi_minus", 0.0);
        for (int j = 0; j < 4; j++) {
            m[8 + j] = -m[8 + j];
            m[12 + j] = -m[12 + j];
        }
        return m;
    }
    if (which == "phi_plus") return {s, o, s, o, o, s, o, s, o, s, o, ns, s, o, ns, o};  // gates.rs:264-274
    fail(kValueError, "unknown dense gate " + which);
}

std::vector<uint64_t> Operation::touched() const {
    switch (type) {
        case One:
        case X: {
            std::vector<uint64_t> q;
            for (auto& c : controls) q.push_back(c.qubit);
            q.push_back(target);
            return q;
        }
        case Swap: {
            std::vector<uint64_t> q;
            for (auto& c : controls) q.push_back(c.qubit);
            q.push_back(a);
            q.push_back(b);
            return q;
        }
        case Diagonal:
        case Dense: return qubits;
        case Measure:
        case Reset: return {qubit};
        case Conditional: return inner->touched();
        case Noop: return {};
    }
    return {};
}

bool gate_matrix_1q(const Instruction& in, uint64_t* qubit, Mat2* m) {
    const double* p = in.p;
    switch (in.kind) {
        case Kind::Id: case Kind::U0: *m = kI; break;
        case Kind::X: *m = kX; break;
        case Kind::Y: *m = kY; break;
        case Kind::Z: *m = kZ; break;
        case Kind::H: *m = g_h(); break;
        case Kind::S: *m = g_s(); break;
        case Kind::Sdg: *m = g_sdg(); break;
        case Kind::T: *m = g_t(); break;
        case Kind::Tdg: *m = g_tdg(); break;
        case Kind::Sx: *m = g_sx(); break;
        case Kind::Sxdg: *m = g_sxdg(); break;
        case Kind::U3: case Kind::U: *m = g_u3(p[kTheta], p[kPhi], p[kLam]); break;
        case Kind::U2: *m = g_u2(p[kPhi], p[kLam]); break;
        case Kind::U1: case Kind::P: *m = g_p(p[kLam]); break;
        case Kind::Rx: *m = g_rx(p[kTheta]); break;
        case Kind::Ry: *m = g_ry(p[kTheta]); break;
        case Kind::Rz: *m = g_rz(p[kPhi]); break;
        default: return false;
    }
    *qubit = in.qubits[0];
    return true;
}

bool compile_instruction(const Instruction& in, Operation* out) {
    uint64_t q;
    Mat2 m;
    if (gate_matrix_1q(in, &q, &m)) {
        *out = op_one(q, m, {});
        return true;
    }
    const double* p = in.p;
    const auto& qs = in.qubits;
    auto controlled = [&](const Mat2& u) { return op_one(qs[1], u, {{qs[0], true}}); };
    switch (in.kind) {
        case Kind::Cx: *out = controlled(kX); return true;
        case Kind::Cy: *out = controlled(kY); return true;
        case Kind::Cz: *out = controlled(kZ); return true;
        case Kind::Ch: *out = controlled(g_h()); return true;
        case Kind::Csx: *out = controlled(g_sx()); return true;
        case Kind::Crx: *out = controlled(g_rx(p[kTheta])); return true;
        case Kind::Cry: *out = controlled(g_ry(p[kTheta])); return true;
        case Kind::Crz: *out = controlled(g_rz(p[kLam])); return true;
        case Kind::Cu1: case Kind::Cp: *out = controlled(g_p(p[kLam])); return true;
        case Kind::Cu3: *out = controlled(g_u3(p[kTheta], p[kPhi], p[kLam])); return true;
        case Kind::Cu: {
            Mat2 u = g_u3(p[kTheta], p[kPhi], p[kLam]);
            cplx phase(std::cos(p[kGamma]), std::sin(p[kGamma]));
            for (auto& row : u)
                for (auto& v : row) v = v * phase;
            *out = controlled(u);
            return true;
        }
        case Kind::Swap: *out = op_swap(qs[0], qs[1], {}); return true;
        case Kind::Cswap: *out = op_swap(qs[1], qs[2], {{qs[0], true}}); return true;
        case Kind::Ccx: *out = op_x(qs[2], {{qs[0], true}, {qs[1], true}}); return true;
        case Kind::C3x: *out = op_x(qs[3], {{qs[0], true}, {qs[1], true}, {qs[2], true}}); return true;
        case Kind::C4x: *out = op_x(qs[4], {{qs[0], true}, {qs[1], true}, {qs[2], true}, {qs[3], true}}); return true;
        case Kind::C3sqrtx: *out = op_one(qs[3], g_sx(), {{qs[0], true}, {qs[1], true}, {qs[2], true}}); return true;
        case Kind::Rxx: *out = op_dense(qs, gate_matrix_dense("rxx", p[kTheta])); return true;
        case Kind::Rzz: *out = op_dense(qs, gate_matrix_dense("rzz", p[kTheta])); return true;
        case Kind::Rccx: *out = op_dense(qs, gate_matrix_dense("rccx", 0)); return true;
        case Kind::Rc3x: *out = op_dense(qs, gate_matrix_dense("rc3x", 0)); return true;
        case Kind::Measure:
            out->type = Operation::Measure;
            out->qubit = qs[0];
            out->cbit = in.cbit;
            return true;
        case Kind::Reset:
            out->type = Operation::Reset;
            out->qubit = qs[0];
            return true;
        case Kind::Conditional: {
            Operation inner;
            if (!compile_instruction(*in.op, &inner)) inner.type = Operation::Noop;
            out->type = Operation::Conditional;
            out->condition = in.condition;
            out->inner = std::make_shared<Operation>(std::move(inner));
            return true;
        }
        case Kind::Barrier: return false;
        case Kind::Gate: {
            std::string nm = lower(in.name);
            if (nm == "remote_link_phi_plus" || nm == "remote_epr" || nm == "epr") {
                *out = op_dense(qs, gate_matrix_dense("phi_plus", 0));
                return true;
            }
            if (nm == "remote_link_psi_plus") {
                *out = op_dense(qs, gate_matrix_dense("psi_plus", 0));
                return true;
            }
            if (nm == "remote_link_psi_minus") {
                *out = op_dense(qs, gate_matrix_dense("psi_minus", 0));
                return true;
            }
            if (nm == "nonlocal_cz" || nm == "remote_cz") {
                *out = controlled(kZ);
                return true;
            }
            if (nm == "remote_cx") {
                *out = controlled(kX);
                return true;
            }
            if (nm == "remote_rzz") {
                *out = op_dense(qs, gate_matrix_dense("rzz", in.params[0]));
                return true;
            }
            if (nm == "remote_cu1") {
                *out = controlled(g_p(in.params[0]));
                return true;
            }
            if (nm == "remote_barrier") return false;
            fail(kValueError, "Unsupported generic gate \"" + in.name + "\"; decompose it before simulating");
        }
        default: fail(kValueError, std::string("Unsupported instruction ") + kind_name(in.kind));
    }
}

// compile, execution.rs:368-416.  std::map iterates in ascending qubit order
// like the reference's BTreeMap.
std::vector<Operation> compile(const std::vector<Instruction>& instructions) {
    std::map<uint64_t, Mat2> pending;
    std::vector<Operation> result;
    auto flush = [&](uint64_t q) {
        auto it = pending.find(q);
        if (it == pending.end()) return;
        Mat2 m = it->second;
        pending.erase(it);
        if (m != kI) result.push_back(op_one(q, m, {}));
    };
    for (const Instruction& in : instructions) {
        uint64_t q;
        Mat2 m;
        if (gate_matrix_1q(in, &q, &m)) {
            auto it = pending.find(q);
            Mat2 old = it == pending.end() ? kI : it->second;
            Mat2 prod;
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++) {
                    cplx acc(0, 0);
                    for (int k = 0; k < 2; k++) acc = acc + m[i][k] * old[k][j];
                    prod[i][j] = acc;
                }
            pending[q] = prod;
            continue;
        }
        std::vector<uint64_t> touched;
        if (in.kind == Kind::Barrier || in.kind == Kind::Measure) {
            for (auto& kv : pending) touched.push_back(kv.first);
        } else {
            touched = in.operands();
        }
        for (uint64_t t : touched) flush(t);
        Operation op;
        if (compile_instruction(in, &op)) result.push_back(std::move(op));
    }
    std::vector<uint64_t> rest;
    for (auto& kv : pending) rest.push_back(kv.first);
    for (uint64_t t : rest) flush(t);
    return result;
}

namespace {
void hexd(std::string& s, double v) {
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    char buf[24];
    std::snprintf(buf, sizeof buf, "\"%016llx\"", static_cast<unsigned long long>(bits));
    s += buf;
}
void hexc(std::string& s, cplx c) {
    s += "[";
    hexd(s, c.re);
    s += ",";
    hexd(s, c.im);
    s += "]";
}
void dump_controls(std::string& s, const std::vector<Control>& cs) {
    s += "[";
    for (size_t i = 0; i < cs.size(); i++) {
        if (i) s += ",";
        s += "[" + std::to_string(cs[i].qubit) + "," + (cs[i].value ? "1" : "0") + "]";
    }
    s += "]";
}
void dump_one(std::string& s, const Operation& op) {
    switch (op.type) {
        case Operation::One:
            s += "{\"op\":\"one\",\"target\":" + std::to_string(op.target) + ",\"controls\":";
            dump_controls(s, op.controls);
            s += ",\"m\":[";
            hexc(s, op.m[0][0]);
            s += ",";
            hexc(s, op.m[0][1]);
            s += ",";
            hexc(s, op.m[1][0]);
            s += ",";
            hexc(s, op.m[1][1]);
            s += "]}";
            break;
        case Operation::X:
            s += "{\"op\":\"x\",\"target\":" + std::to_string(op.target) + ",\"controls\":";
            dump_controls(s, op.controls);
            s += "}";
            break;
        case Operation::Swap:
            s += "{\"op\":\"swap\",\"a\":" + std::to_string(op.a) + ",\"b\":" + std::to_string(op.b) + ",\"controls\":";
            dump_controls(s, op.controls);
            s += "}";
            break;
        case Operation::Diagonal:
        case Operation::Dense: {
            s += op.type == Operation::Diagonal ? "{\"op\":\"diag\",\"qubits\":[" : "{\"op\":\"dense\",\"qubits\":[";
            for (size_t i = 0; i < op.qubits.size(); i++) s += (i ? "," : "") + std::to_string(op.qubits[i]);
            s += "],\"values\":[";
            for (size_t i = 0; i < op.values.size(); i++) {
                if (i) s += ",";
                hexc(s, op.values[i]);
            }
            s += "]}";
            break;
        }
        case Operation::Measure:
            s += "{\"op\":\"measure\",\"qubit\":" + std::to_string(op.qubit) + ",\"cbit\":" + std::to_string(op.cbit) + "}";
            break;
        case Operation::Reset: s += "{\"op\":\"reset\",\"qubit\":" + std::to_string(op.qubit) + "}"; break;
        case Operation::Noop: s += "{\"op\":\"noop\"}"; break;
        case Operation::Conditional:
            s += "{\"op\":\"cond\",\"condition\":[" + std::to_string(op.condition.creg_base) + "," +
                 std::to_string(op.condition.creg_size) + "," + std::to_string(op.condition.creg_value) + "],\"inner\":";
            dump_one(s, *op.inner);
            s += "}";
            break;
    }
}
}  // namespace

std::string dump_operations(const std::vector<Operation>& ops) {
    std::string s = "[";
    for (size_t i = 0; i < ops.size(); i++) {
        if (i) s += ",";
        dump_one(s, ops[i]);
    }
    s += "]";
    return s;
}

}  // namespace dq

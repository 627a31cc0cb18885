"""CPU oracle for the dense statevector path of dqsim 0.1.2.

TEST INFRASTRUCTURE ONLY.  It restates, on the CPU and in complex128, what the
reference's ``StatevectorSimulator`` does, so that the CUDA product can be
checked against it and a CPU baseline can be timed beside it.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may import it; the
product never does.

Pinning: the reference is Rust/PyO3 and cannot be built in this environment, so
this restatement is pinned by the known-answer tests in the reference's own
test suites (src/engine.rs:509-779, src/gates.rs:302-378,
src/monolithic/statevector/shots.rs:262-308,
src/monolithic/statevector/validation.rs:14-200 and
tests/test_statevector.py:53-347), ported in tests/test_oracle_*.py.  Exact
seeded counts depend on rand_chacha's ChaCha8 stream, restated in sv_oracle.c;
the block function is pinned against ChaCha20 from ``cryptography``, the seed
expansion is not pinned by any reference output.

Layout: the front end (JSON transport, validation, gate tables, 1q fusion,
shot strategies) is Python and follows the reference line by line; the hot
loops are C (``libsv_oracle.so``, OpenMP) and follow ``src/engine.rs``.
"""

from __future__ import annotations

import ctypes
import json
import math
import os
import secrets
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "libsv_oracle.so"
_lib = None

U64 = (1 << 64) - 1
USIZE_BITS = 64
ISIZE_MAX = (1 << 63) - 1


def build():
    """Compile libsv_oracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        P = ctypes.c_void_p
        i, d, u64 = ctypes.c_int, ctypes.c_double, ctypes.c_uint64
        L.orc_apply_one_qubit.argtypes = [P, i, i, P, P, P, i, i, i]
        L.orc_apply_diagonal.argtypes = [P, i, P, i, P, i]
        L.orc_apply_swap.argtypes = [P, i, i, i, P, P, i, i]
        L.orc_apply_dense.argtypes = [P, i, P, i, P, i]
        L.orc_measure.argtypes = [P, i, i, d, i, P]
        L.orc_measure.restype = i
        L.orc_marginal_probs.argtypes = [P, i, P, i, P]
        L.orc_fidelity.argtypes = [P, P, u64]
        L.orc_fidelity.restype = d
        L.orc_cdf_inplace.argtypes = [P, u64]
        L.orc_cdf_inplace.restype = i
        L.orc_partition_point.argtypes = [P, u64, d]
        L.orc_partition_point.restype = u64
        L.orc_chacha_block_words.argtypes = [P, i, P]
        L.orc_seed_from_u64.argtypes = [u64, P]
        L.orc_chacha8_u64.argtypes = [u64, u64]
        L.orc_chacha8_u64.restype = u64
        L.orc_chacha8_f64.argtypes = [u64, u64]
        L.orc_chacha8_f64.restype = d
        L.orc_u64_to_f64.argtypes = [u64]
        L.orc_u64_to_f64.restype = d
        L.orc_first_draws.argtypes = [u64, u64, u64, P]
        L.orc_stream_draws.argtypes = [u64, u64, u64, P]
        L.orc_num_threads.restype = i
        L.orc_set_num_threads.argtypes = [i]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ints(xs):
    return np.ascontiguousarray(np.asarray(list(xs), dtype=np.int32))


def _cplx(xs):
    return np.ascontiguousarray(np.asarray(xs, dtype=np.complex128))


# ---------------------------------------------------------------------------
# RNG (rand_chacha ChaCha8Rng::seed_from_u64, rand 0.8 Standard f64)
# ---------------------------------------------------------------------------
class ChaCha8Stream:
    """Sequential f64 draws of ChaCha8Rng::seed_from_u64(seed)."""

    def __init__(self, seed):
        self.seed = seed & U64
        self.k = 0

    def gen_f64(self):
        v = lib().orc_chacha8_f64(self.seed, self.k)
        self.k += 1
        return v


def first_draws(seed, count, start=0):
    out = np.empty(count, dtype=np.float64)
    if count:
        lib().orc_first_draws(seed & U64, start, count, _ptr(out))
    return out


def stream_draws(seed, count, start=0):
    out = np.empty(count, dtype=np.float64)
    if count:
        lib().orc_stream_draws(seed & U64, start, count, _ptr(out))
    return out


# ---------------------------------------------------------------------------
# JSON transport, src/types.rs:7-296 (serde, internally tagged by "kind")
# ---------------------------------------------------------------------------
class CircuitError(ValueError):
    pass


USZ, F64, U64T, STR, USZLIST, F64LIST, OP, COND = range(8)

_SCHEMA = {
    # Single-qubit fixed, types.rs:66-98
    **{k: {"qubit": USZ} for k in ("id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "u0")},
    # Single-qubit parametric, types.rs:102-141
    "u3": {"qubit": USZ, "theta": F64, "phi": F64, "lam": F64},
    "u2": {"qubit": USZ, "phi": F64, "lam": F64},
    "u1": {"qubit": USZ, "lam": F64},
    "u": {"qubit": USZ, "theta": F64, "phi": F64, "lam": F64},
    "p": {"qubit": USZ, "lam": F64},
    "rx": {"qubit": USZ, "theta": F64},
    "ry": {"qubit": USZ, "theta": F64},
    "rz": {"qubit": USZ, "phi": F64},
    # Two-qubit, types.rs:145-221
    **{k: {"control": USZ, "target": USZ} for k in ("cx", "cz", "cy", "ch", "csx")},
    "swap": {"a": USZ, "b": USZ},
    "crx": {"control": USZ, "target": USZ, "theta": F64},
    "cry": {"control": USZ, "target": USZ, "theta": F64},
    "crz": {"control": USZ, "target": USZ, "lam": F64},
    "cu1": {"control": USZ, "target": USZ, "lam": F64},
    "cp": {"control": USZ, "target": USZ, "lam": F64},
    "cu3": {"control": USZ, "target": USZ, "theta": F64, "phi": F64, "lam": F64},
    "cu": {"control": USZ, "target": USZ, "theta": F64, "phi": F64, "lam": F64, "gamma": F64},
    "rxx": {"a": USZ, "b": USZ, "theta": F64},
    "rzz": {"a": USZ, "b": USZ, "theta": F64},
    # Three+ qubits, types.rs:225-264
    "ccx": {"control1": USZ, "control2": USZ, "target": USZ},
    "cswap": {"control": USZ, "target1": USZ, "target2": USZ},
    "rccx": {"control1": USZ, "control2": USZ, "target": USZ},
    "rc3x": {"control1": USZ, "control2": USZ, "control3": USZ, "target": USZ},
    "c3x": {"control1": USZ, "control2": USZ, "control3": USZ, "target": USZ},
    "c3sqrtx": {"control1": USZ, "control2": USZ, "control3": USZ, "target": USZ},
    "c4x": {"control1": USZ, "control2": USZ, "control3": USZ, "control4": USZ, "target": USZ},
    # Generic, measurement, control, no-ops, types.rs:268-295
    "gate": {"name": STR, "params": F64LIST, "qubits": USZLIST},
    "measure": {"qubit": USZ, "cbit": USZ},
    "reset": {"qubit": USZ},
    "conditional": {"condition": COND, "op": OP},
    "barrier": {},
    "classical": {"name": STR},
}

# Operand order of Instruction::qubits, types.rs:346-463
_QUBIT_FIELDS = {
    "swap": ("a", "b"), "rxx": ("a", "b"), "rzz": ("a", "b"),
    "ccx": ("control1", "control2", "target"), "rccx": ("control1", "control2", "target"),
    "cswap": ("control", "target1", "target2"),
    "rc3x": ("control1", "control2", "control3", "target"),
    "c3x": ("control1", "control2", "control3", "target"),
    "c3sqrtx": ("control1", "control2", "control3", "target"),
    "c4x": ("control1", "control2", "control3", "control4", "target"),
}
for _k in ("cx", "cz", "cy", "ch", "csx", "crx", "cry", "crz", "cu1", "cp", "cu3", "cu"):
    _QUBIT_FIELDS[_k] = ("control", "target")


def _is_int(v):
    return isinstance(v, int) and not isinstance(v, bool)


def _check(value, kind, where):
    if kind == USZ or kind == U64T:
        if not _is_int(value) or value < 0 or value > U64:
            raise CircuitError(f"invalid unsigned integer for {where}")
        return value
    if kind == F64:
        if isinstance(value, bool) or not isinstance(value, (int, float)):
            raise CircuitError(f"invalid number for {where}")
        return float(value)
    if kind == STR:
        if not isinstance(value, str):
            raise CircuitError(f"invalid string for {where}")
        return value
    if kind == USZLIST:
        if not isinstance(value, list):
            raise CircuitError(f"invalid sequence for {where}")
        return [_check(v, USZ, where) for v in value]
    if kind == F64LIST:
        if not isinstance(value, list):
            raise CircuitError(f"invalid sequence for {where}")
        return [_check(v, F64, where) for v in value]
    if kind == OP:
        return parse_instruction(value)
    if kind == COND:
        if not isinstance(value, dict):
            raise CircuitError("invalid condition")
        return {
            "creg_base": _check(_req(value, "creg_base"), USZ, "creg_base"),
            "creg_size": _check(_req(value, "creg_size"), USZ, "creg_size"),
            "creg_value": _check(_req(value, "creg_value"), U64T, "creg_value"),
        }
    raise AssertionError(kind)


def _req(obj, key):
    if key not in obj:
        raise CircuitError(f"missing field `{key}`")
    return obj[key]


def parse_instruction(obj):
    if not isinstance(obj, dict):
        raise CircuitError("instruction must be an object")
    kind = _req(obj, "kind")
    if not isinstance(kind, str) or kind not in _SCHEMA:
        raise CircuitError(f"unknown variant {kind!r}")
    out = {"kind": kind}
    for field, ftype in _SCHEMA[kind].items():
        out[field] = _check(_req(obj, field), ftype, field)
    return out


def _reject_constant(name):
    raise CircuitError(f"invalid JSON constant {name}")


def parse_circuit(text):
    """serde_json::from_str::<Circuit>, types.rs:15-21."""
    try:
        data = json.loads(text, parse_constant=_reject_constant)
    except CircuitError:
        raise
    except Exception as exc:  # noqa: BLE001 - any malformed JSON is a parse error
        raise CircuitError(f"Circuit JSON parse error: {exc}") from None
    if not isinstance(data, dict):
        raise CircuitError("Circuit JSON parse error: expected an object")

    def regs(v):
        if not isinstance(v, dict):
            raise CircuitError("registers must be a map")
        out = {}
        for name, r in v.items():
            if not isinstance(r, dict):
                raise CircuitError("register must be an object")
            out[name] = {
                "name": _check(_req(r, "name"), STR, "name"),
                "size": _check(_req(r, "size"), USZ, "size"),
                "base": _check(_req(r, "base"), USZ, "base"),
            }
        return out

    qregs = regs(_req(data, "qregs"))
    cregs = regs(data.get("cregs", {}))
    insts = _req(data, "instructions")
    if not isinstance(insts, list):
        raise CircuitError("instructions must be a sequence")
    return {"qregs": qregs, "cregs": cregs, "instructions": [parse_instruction(i) for i in insts]}


def num_qubits(c):
    """Circuit::num_qubits, types.rs:24-30 (base + size wraps like usize)."""
    return max(((r["base"] + r["size"]) & U64 for r in c["qregs"].values()), default=0)


def num_cbits(c):
    return max(((r["base"] + r["size"]) & U64 for r in c["cregs"].values()), default=0)


def inst_qubits(inst):
    """Instruction::qubits, types.rs:346-463."""
    k = inst["kind"]
    if k in ("barrier", "classical"):
        return []
    if k == "gate":
        return list(inst["qubits"])
    if k == "conditional":
        return inst_qubits(inst["op"])
    if k in _QUBIT_FIELDS:
        return [inst[f] for f in _QUBIT_FIELDS[k]]
    return [inst["qubit"]]


# ---------------------------------------------------------------------------
# Validation, src/validation.rs:5-182 and statevector/validation.rs:3-12
# ---------------------------------------------------------------------------
_GENERIC = {
    "remote_link_phi_plus": (2, 0), "remote_link_psi_minus": (2, 0), "remote_link_psi_plus": (2, 0),
    "nonlocal_cz": (2, 0), "remote_cz": (2, 0), "remote_cx": (2, 0), "remote_epr": (2, 0),
    "epr": (2, 0), "remote_rzz": (2, 1), "remote_cu1": (2, 1), "remote_barrier": (None, 0),
}


def register_ranges(regs, kind):
    ranges = []
    for name, r in regs.items():
        end = r["base"] + r["size"]
        if end > U64:
            raise CircuitError(f"{kind} register {name!r} has an overflowing range")
        if r["size"] != 0:
            ranges.append((r["base"], end))
    ranges.sort()
    for a, b in zip(ranges, ranges[1:]):
        if b[0] < a[1]:
            raise CircuitError(f"Overlapping {kind} registers")
    return ranges


def _declared(i, ranges):
    return any(s <= i < e for s, e in ranges)


def _finite(*xs):
    return all(math.isfinite(x) for x in xs)


def validate_instruction(inst, qubits, cbits):
    k = inst["kind"]
    if k == "conditional":
        c = inst["condition"]
        if c["creg_size"] == 0 or c["creg_size"] > 64:
            raise CircuitError("Condition width must be between 1 and 64 bits")
        end = c["creg_base"] + c["creg_size"]
        if end > U64:
            raise CircuitError("Condition has an overflowing classical range")
        for bit in range(c["creg_base"], end):
            if not _declared(bit, cbits):
                raise CircuitError("Condition refers to undeclared classical bits")
        if c["creg_size"] < 64 and c["creg_value"] >= (1 << c["creg_size"]):
            raise CircuitError("Condition value does not fit its classical width")
        return validate_instruction(inst["op"], qubits, cbits)
    ops = inst_qubits(inst)
    for idx, q in enumerate(ops):
        if not _declared(q, qubits):
            raise CircuitError(f"Qubit {q} is not declared by a quantum register")
        if q in ops[:idx]:
            raise CircuitError(f"Gate operands must be distinct; qubit {q} is repeated")
    if k == "measure" and not _declared(inst["cbit"], cbits):
        raise CircuitError(f"Classical bit {inst['cbit']} is not declared by a classical register")
    if k == "classical":
        raise CircuitError(f"Unsupported classical operation: {inst['name']!r}")
    if k == "gate":
        name = inst["name"].lower()
        if name not in _GENERIC:
            raise CircuitError(f"Unsupported generic gate: {inst['name']!r}. Decompose it before simulating.")
        arity, nparams = _GENERIC[name]
        if arity is not None and len(inst["qubits"]) != arity:
            raise CircuitError(f"Gate requires {arity} qubits")
        if len(inst["params"]) != nparams:
            raise CircuitError(f"Gate requires {nparams} parameters")
    fin = True
    if k in ("u3", "u", "cu3"):
        fin = _finite(inst["theta"], inst["phi"], inst["lam"])
    elif k == "cu":
        fin = _finite(inst["theta"], inst["phi"], inst["lam"], inst["gamma"])
    elif k == "u2":
        fin = _finite(inst["phi"], inst["lam"])
    elif k in ("u1", "p", "crz", "cu1", "cp"):
        fin = _finite(inst["lam"])
    elif k in ("rx", "ry", "crx", "cry", "rxx", "rzz"):
        fin = _finite(inst["theta"])
    elif k == "rz":
        fin = _finite(inst["phi"])
    elif k == "gate":
        fin = _finite(*inst["params"])
    if not fin:
        raise CircuitError("Gate parameters must be finite numbers")
    if k in ("u3", "u2", "u", "cu3", "cu") and not math.isfinite(inst["phi"] + inst["lam"]):
        raise CircuitError("The combined phase phi + lam must be finite")


def validate_circuit(c):
    qubits = register_ranges(c["qregs"], "quantum")
    cbits = register_ranges(c["cregs"], "classical")
    for index, inst in enumerate(c["instructions"]):
        try:
            validate_instruction(inst, qubits, cbits)
        except CircuitError as e:
            raise CircuitError(f"Instruction {index}: {e}") from None
    if num_qubits(c) >= USIZE_BITS:
        raise CircuitError(f"Statevector qubit count must be less than {USIZE_BITS}")


# ---------------------------------------------------------------------------
# Gate matrices, src/gates.rs:23-274 and gate_matrix_1q, src/types.rs:303-344
# ---------------------------------------------------------------------------
def C(re, im=0.0):
    return complex(float(re), float(im))


S2 = 0.7071067811865476  # FRAC_1_SQRT_2
X = [[C(0), C(1)], [C(1), C(0)]]
Y = [[C(0), C(0, -1)], [C(0, 1), C(0)]]
Z = [[C(1), C(0)], [C(0), C(-1)]]
I2 = [[C(1), C(0)], [C(0), C(1)]]


def h():
    return [[C(S2), C(S2)], [C(S2), C(-S2)]]


def s_gate():
    return [[C(1), C(0)], [C(0), C(0, 1)]]


def sdg():
    return [[C(1), C(0)], [C(0), C(0, -1)]]


def t_gate():
    return [[C(1), C(0)], [C(0), C(S2, S2)]]


def tdg():
    return [[C(1), C(0)], [C(0), C(S2, -S2)]]


def sx():
    a, b = C(0.5, 0.5), C(0.5, -0.5)
    return [[a, b], [b, a]]


def sxdg():
    a, b = C(0.5, -0.5), C(0.5, 0.5)
    return [[a, b], [b, a]]


def u3(theta, phi, lam):
    ct, st = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return [
        [C(ct), -(C(math.cos(lam), math.sin(lam)) * C(st))],
        [C(math.cos(phi), math.sin(phi)) * C(st), C(math.cos(phi + lam), math.sin(phi + lam)) * C(ct)],
    ]


def u2(phi, lam):
    return u3(math.pi / 2.0, phi, lam)


def p(lam):
    return [[C(1), C(0)], [C(0), C(math.cos(lam), math.sin(lam))]]


def rx(theta):
    c2, s2 = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return [[C(c2), C(0, -s2)], [C(0, -s2), C(c2)]]


def ry(theta):
    c2, s2 = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return [[C(c2), C(-s2)], [C(s2), C(c2)]]


def rz(phi):
    return [[C(math.cos(-phi / 2.0), math.sin(-phi / 2.0)), C(0)],
            [C(0), C(math.cos(phi / 2.0), math.sin(phi / 2.0))]]


def rxx(theta):
    cv, sv = math.cos(theta / 2.0), math.sin(theta / 2.0)
    o, m = C(0), C(0, -sv)
    return [[C(cv), o, o, m], [o, C(cv), m, o], [o, m, C(cv), o], [m, o, o, C(cv)]]


def rzz(theta):
    ep = C(math.cos(theta / 2.0), math.sin(theta / 2.0))
    em = C(math.cos(theta / 2.0), -math.sin(theta / 2.0))
    o = C(0)
    return [[em, o, o, o], [o, ep, o, o], [o, o, ep, o], [o, o, o, em]]


def _identity(n):
    return [[C(1) if i == j else C(0) for j in range(n)] for i in range(n)]


def rccx():
    m = _identity(8)
    m[5][5] = C(-1)
    m[6][6] = C(0)
    m[7][7] = C(0)
    m[6][7] = C(0, -1)
    m[7][6] = C(0, 1)
    return m


def rc3x():
    m = _identity(16)
    m[12][12] = C(0, 1)
    m[13][13] = C(0, -1)
    m[14][14] = C(0)
    m[15][15] = C(0)
    m[14][15] = C(1)
    m[15][14] = C(-1)
    return m


def psi_minus():
    s, o = C(S2), C(0)
    return [[o, s, o, s], [s, o, s, o], [C(-S2), o, s, o], [o, C(-S2), o, s]]


def psi_plus():
    pm = psi_minus()
    return [pm[0][:], pm[1][:], [-v for v in pm[2]], [-v for v in pm[3]]]


def phi_plus():
    s, o = C(S2), C(0)
    return [[s, o, s, o], [o, s, o, s], [o, s, o, C(-S2)], [s, o, C(-S2), o]]


def gate_matrix_1q(inst):
    k = inst["kind"]
    if k in ("id", "u0"):
        return inst["qubit"], I2
    table = {"x": lambda: X, "y": lambda: Y, "z": lambda: Z, "h": h, "s": s_gate, "sdg": sdg,
             "t": t_gate, "tdg": tdg, "sx": sx, "sxdg": sxdg}
    if k in table:
        return inst["qubit"], table[k]()
    if k in ("u3", "u"):
        return inst["qubit"], u3(inst["theta"], inst["phi"], inst["lam"])
    if k == "u2":
        return inst["qubit"], u2(inst["phi"], inst["lam"])
    if k in ("u1", "p"):
        return inst["qubit"], p(inst["lam"])
    if k == "rx":
        return inst["qubit"], rx(inst["theta"])
    if k == "ry":
        return inst["qubit"], ry(inst["theta"])
    if k == "rz":
        return inst["qubit"], rz(inst["phi"])
    return None


# ---------------------------------------------------------------------------
# Operation lowering and 1q fusion, src/monolithic/statevector/execution.rs:21-416
# Operations are tuples:
#   ("one", target, m2, controls)   ("x", target, controls)
#   ("swap", a, b, controls)        ("diag", qubits, diagonal)
#   ("dense", qubits, matrix)       ("measure", qubit, cbit)
#   ("reset", qubit)                ("cond", (base, size, value), op)
# controls are tuples of (qubit, bool).
# ---------------------------------------------------------------------------
ZERO = C(0)


def op_one(target, m, controls):
    """Operation::one, execution.rs:66-87."""
    if m == X:
        return ("x", target, tuple(controls))
    if m[0][1] == ZERO and m[1][0] == ZERO:
        qubits = [q for q, _ in controls] + [target]
        diag = [C(1)] * (1 << len(qubits))
        index = 0
        for _, on in controls:
            index = (index << 1) | int(on)
        index <<= 1
        diag[index] = m[0][0]
        diag[index + 1] = m[1][1]
        return ("diag", tuple(qubits), tuple(diag))
    return ("one", target, tuple(tuple(r) for r in m), tuple(controls))


def op_dense(qubits, m):
    """Operation::dense, execution.rs:89-106."""
    n = len(m)
    if all(i == j or m[i][j] == ZERO for i in range(n) for j in range(n)):
        return ("diag", tuple(qubits), tuple(m[i][i] for i in range(n)))
    return ("dense", tuple(qubits), tuple(tuple(r) for r in m))


def compile_instruction(inst):
    """Operation::compile, execution.rs:108-274."""
    g = gate_matrix_1q(inst)
    if g is not None:
        return op_one(g[0], g[1], [])
    k = inst["kind"]

    def ctl(m):
        return op_one(inst["target"], m, [(inst["control"], True)])

    if k == "cx":
        return ctl(X)
    if k == "cy":
        return ctl(Y)
    if k == "cz":
        return ctl(Z)
    if k == "ch":
        return ctl(h())
    if k == "csx":
        return ctl(sx())
    if k == "crx":
        return ctl(rx(inst["theta"]))
    if k == "cry":
        return ctl(ry(inst["theta"]))
    if k == "crz":
        return ctl(rz(inst["lam"]))
    if k in ("cu1", "cp"):
        return ctl(p(inst["lam"]))
    if k == "cu3":
        return ctl(u3(inst["theta"], inst["phi"], inst["lam"]))
    if k == "cu":
        m = u3(inst["theta"], inst["phi"], inst["lam"])
        phase = C(math.cos(inst["gamma"]), math.sin(inst["gamma"]))
        m = [[v * phase for v in row] for row in m]
        return ctl(m)
    if k == "swap":
        return ("swap", inst["a"], inst["b"], ())
    if k == "cswap":
        return ("swap", inst["target1"], inst["target2"], ((inst["control"], True),))
    if k == "ccx":
        return ("x", inst["target"], ((inst["control1"], True), (inst["control2"], True)))
    if k == "c3x":
        return ("x", inst["target"], tuple((inst[f"control{i}"], True) for i in (1, 2, 3)))
    if k == "c4x":
        return ("x", inst["target"], tuple((inst[f"control{i}"], True) for i in (1, 2, 3, 4)))
    if k == "c3sqrtx":
        return op_one(inst["target"], sx(), [(inst[f"control{i}"], True) for i in (1, 2, 3)])
    if k == "rxx":
        return op_dense([inst["a"], inst["b"]], rxx(inst["theta"]))
    if k == "rzz":
        return op_dense([inst["a"], inst["b"]], rzz(inst["theta"]))
    if k == "rccx":
        return op_dense([inst["control1"], inst["control2"], inst["target"]], rccx())
    if k == "rc3x":
        return op_dense([inst["control1"], inst["control2"], inst["control3"], inst["target"]], rc3x())
    if k == "measure":
        return ("measure", inst["qubit"], inst["cbit"])
    if k == "reset":
        return ("reset", inst["qubit"])
    if k == "conditional":
        c = inst["condition"]
        return ("cond", (c["creg_base"], c["creg_size"], c["creg_value"]), compile_instruction(inst["op"]))
    if k == "barrier":
        return ("noop",)
    if k == "gate":
        name = inst["name"].lower()
        qs = inst["qubits"]
        if name in ("remote_link_phi_plus", "remote_epr", "epr"):
            return op_dense(qs, phi_plus())
        if name == "remote_link_psi_plus":
            return op_dense(qs, psi_plus())
        if name == "remote_link_psi_minus":
            return op_dense(qs, psi_minus())
        if name in ("nonlocal_cz", "remote_cz"):
            return op_one(qs[1], Z, [(qs[0], True)])
        if name == "remote_cx":
            return op_one(qs[1], X, [(qs[0], True)])
        if name == "remote_rzz":
            return op_dense(qs, rzz(inst["params"][0]))
        if name == "remote_cu1":
            return op_one(qs[1], p(inst["params"][0]), [(qs[0], True)])
        if name == "remote_barrier":
            return ("noop",)
        raise CircuitError(f"Unsupported generic gate {inst['name']!r}; decompose it before simulating")
    raise CircuitError(f"Unsupported instruction {k}")


def compile_ops(instructions):
    """compile, execution.rs:368-416 (BTreeMap order: ascending qubit)."""
    pending = {}
    result = []

    def flush(q):
        m = pending.pop(q, None)
        if m is not None and m != I2:
            result.append(op_one(q, m, []))

    for inst in instructions:
        g = gate_matrix_1q(inst)
        if g is not None:
            q, m = g
            old = pending.get(q, I2)
            prod = [[C(0), C(0)], [C(0), C(0)]]
            for i in range(2):
                for j in range(2):
                    for k in range(2):
                        prod[i][j] = prod[i][j] + m[i][k] * old[k][j]
            pending[q] = prod
        else:
            if inst["kind"] in ("barrier", "measure"):
                touched = sorted(pending)
            else:
                touched = inst_qubits(inst)
            for q in touched:
                flush(q)
            op = compile_instruction(inst)
            if op[0] != "noop":
                result.append(op)
    for q in sorted(pending):
        flush(q)
    return result


def is_unitary(op):
    return op[0] not in ("measure", "reset", "cond")


# ---------------------------------------------------------------------------
# Execution on a host complex128 state (execution.rs:276-366)
# ---------------------------------------------------------------------------
def _split_controls(controls):
    return _ints([q for q, _ in controls]), _ints([1 if v else 0 for _, v in controls])


def apply_op(op, state, n, cbits, rng, parallel=True):
    """Operation::execute; cbits is a list of ints; rng has gen_f64()."""
    L = lib()
    kind = op[0]
    par = 1 if parallel else 0
    if kind == "cond":
        (base, size, value), inner = op[1], op[2]
        actual = 0
        for bit in range(size):
            actual |= (cbits[base + bit] & 1) << bit
        if actual == value:
            apply_op(inner, state, n, cbits, rng, parallel)
        return
    if kind == "noop":
        return
    if kind == "one":
        cq, cv = _split_controls(op[3])
        u = _cplx([op[2][0][0], op[2][0][1], op[2][1][0], op[2][1][1]])
        L.orc_apply_one_qubit(_ptr(state), n, op[1], _ptr(u), _ptr(cq), _ptr(cv), len(cq), 0, par)
    elif kind == "x":
        cq, cv = _split_controls(op[2])
        u = _cplx([0, 1, 1, 0])
        L.orc_apply_one_qubit(_ptr(state), n, op[1], _ptr(u), _ptr(cq), _ptr(cv), len(cq), 1, par)
    elif kind == "swap":
        cq, cv = _split_controls(op[3])
        L.orc_apply_swap(_ptr(state), n, op[1], op[2], _ptr(cq), _ptr(cv), len(cq), par)
    elif kind == "diag":
        qs, d = _ints(op[1]), _cplx(op[2])
        L.orc_apply_diagonal(_ptr(state), n, _ptr(qs), len(qs), _ptr(d), par)
    elif kind == "dense":
        qs = _ints(op[1])
        u = _cplx([v for row in op[2] for v in row])
        L.orc_apply_dense(_ptr(state), n, _ptr(qs), len(qs), _ptr(u), par)
    elif kind in ("measure", "reset"):
        draw = rng.gen_f64()
        outcome = L.orc_measure(_ptr(state), n, op[1], draw, par, None)
        if outcome < 0:
            raise RuntimeError("Cannot measure a state with nonfinite or zero norm")
        if kind == "measure":
            cbits[op[2]] = outcome
        elif outcome == 1:
            u = _cplx([0, 1, 1, 0])
            e = _ints([])
            L.orc_apply_one_qubit(_ptr(state), n, op[1], _ptr(u), _ptr(e), _ptr(e), 0, 1, par)
    else:
        raise AssertionError(kind)


def execute(ops, state, n, cbits, rng, parallel=True):
    for op in ops:
        apply_op(op, state, n, cbits, rng, parallel)


def zero_state(n):
    s = np.zeros(1 << n, dtype=np.complex128)
    s[0] = 1.0
    return s


def marginal_probs(state, n, qubits):
    qs = _ints(qubits)
    out = np.empty(1 << len(qubits), dtype=np.float64)
    lib().orc_marginal_probs(_ptr(state), n, _ptr(qs), len(qs), _ptr(out))
    return out


def cdf_from_probs(probs):
    """Running sums of `probs` normalised in place (shots.rs:137-149 turns the
    marginal table itself into the CDF); None for a nonfinite or zero total."""
    cdf = np.ascontiguousarray(probs, dtype=np.float64)
    if not lib().orc_cdf_inplace(_ptr(cdf), len(cdf)):
        return None
    return cdf


def partition_point(cdf, draw):
    return int(lib().orc_partition_point(_ptr(cdf), len(cdf), float(draw)))


# ---------------------------------------------------------------------------
# Shots, src/monolithic/statevector/shots.rs:22-260
# ---------------------------------------------------------------------------
class BudgetError(MemoryError):
    pass


def state_layout(n):
    if n >= 64:
        raise BudgetError("State dimension overflow")
    length = 1 << n
    nbytes = length * 16
    if nbytes > ISIZE_MAX:
        raise BudgetError("State byte size overflow")
    return length, nbytes


def check_budget(required, budget):
    if required > budget:
        raise BudgetError(
            f"Simulation needs at least {required} working bytes, exceeding max_memory_mb budget ({budget} bytes)")


def format_bits(cbits):
    return "".join(str(b) for b in reversed(cbits))


def run_shots(ops, n, ncb, shots, seed, budget, max_parallel_shots, sample_terminal, threads=None):
    """run_shots, shots.rs:59-260.  Returns a dict like ShotOutput."""
    threads = threads or lib().orc_num_threads()
    empty = {"counts": {}, "strategy": None, "parallel_shots": 0, "working_bytes": 0, "prefix_ops": 0}
    if shots == 0:
        return {**empty, "strategy": "empty"}
    length, state_bytes = state_layout(n)
    worker_bytes = state_bytes + ncb
    check_budget(worker_bytes, budget)
    prefix_end = next((i for i, op in enumerate(ops) if not is_unitary(op)), len(ops))
    terminal = all(op[0] == "measure" for op in ops[prefix_end:])
    if sample_terminal and terminal:
        mapping = {}
        for op in ops[prefix_end:]:
            mapping[op[2]] = op[1]
        if not mapping:
            return {**empty, "strategy": "terminal_sampling", "counts": {"0" * ncb: shots}}
        qubits = sorted(set(mapping.values()), reverse=True)
        shifts = sorted((cbit, len(qubits) - 1 - qubits.index(q)) for cbit, q in mapping.items())
        cdf_bytes = (1 << len(qubits)) * 8
        required = worker_bytes + cdf_bytes
        if required <= budget:
            state = zero_state(n)
            cbits = [0] * ncb
            execute(ops[:prefix_end], state, n, cbits, ChaCha8Stream(seed), True)
            cdf = cdf_from_probs(marginal_probs(state, n, qubits))
            if cdf is None:
                raise RuntimeError("Invalid state normalization when sampling")
            del state  # shots.rs:150
            draws = first_draws(seed, shots)
            idx = np.searchsorted(cdf, draws, side="right")
            idx = np.minimum(idx, len(cdf) - 1)
            uniq, cnt = np.unique(idx, return_counts=True)
            counts = {}
            for i, c in zip(uniq.tolist(), cnt.tolist()):
                for cbit, shift in shifts:
                    cbits[cbit] = (i >> shift) & 1
                key = format_bits(cbits)
                counts[key] = counts.get(key, 0) + c
            return {"counts": counts, "strategy": "terminal_sampling", "parallel_shots": 1,
                    "working_bytes": required, "prefix_ops": prefix_end}
    cache_prefix = shots > 1 and prefix_end > 0 and state_bytes <= budget - worker_bytes
    prefix_bytes = state_bytes if cache_prefix else 0
    workers = max(1, min(shots, max_parallel_shots or threads, threads, (budget - prefix_bytes) // worker_bytes))
    prefix = None
    if cache_prefix:
        prefix = zero_state(n)
        execute(ops[:prefix_end], prefix, n, [0] * ncb, ChaCha8Stream(seed), True)
    tail = ops[prefix_end:] if cache_prefix else ops
    counts = {}
    for shot in range(shots):
        state = prefix.copy() if prefix is not None else zero_state(n)
        cbits = [0] * ncb
        execute(tail, state, n, cbits, ChaCha8Stream(seed + shot), workers == 1)
        key = format_bits(cbits)
        counts[key] = counts.get(key, 0) + 1
    return {"counts": counts, "strategy": "trajectories", "parallel_shots": workers,
            "working_bytes": prefix_bytes + workers * worker_bytes,
            "prefix_ops": prefix_end if cache_prefix else 0}


# ---------------------------------------------------------------------------
# Python-facing mirror of StatevectorSimulator / SimulationResult
# (src/monolithic/statevector/simulator.rs:85-372)
# ---------------------------------------------------------------------------
def _validate_query(qubits, n):
    for i, q in enumerate(qubits):
        if q >= n or q in qubits[:i]:
            raise ValueError("Query qubits must be distinct and within the statevector's range")


def sample_counts(state, n, shots, rng_seed, qubits=None):
    """sample_counts, engine.rs:457-507 (one ChaCha8 stream for all shots)."""
    q = list(range(n - 1, -1, -1)) if qubits is None else list(qubits)
    if shots == 0:
        return {}
    cdf = marginal_probs(state, n, q)
    total = 0.0
    for v in cdf.tolist():
        total += v
    if not math.isfinite(total) or total <= 0.0:
        raise RuntimeError("Cannot sample a state with nonfinite or zero norm")
    cum = 0.0
    out = np.empty_like(cdf)
    for i, v in enumerate(cdf.tolist()):
        cum += v
        out[i] = min(cum / total, 1.0)
    out[-1] = 1.0
    draws = stream_draws(rng_seed, shots)
    idx = np.searchsorted(out, draws, side="right")
    uniq, cnt = np.unique(idx, return_counts=True)
    res = {}
    for i, c in zip(uniq.tolist(), cnt.tolist()):
        key = format(i, f"0{len(q)}b") if q else ""
        res[key] = c
    return res


class OracleResult:
    def __init__(self, state, n, cbits):
        self.state = state
        self.num_qubits = n
        self.classical_bits = {i: b for i, b in enumerate(cbits)}

    @property
    def statevector(self):
        return self.state.copy()

    def probabilities(self, qubits=None):
        n = self.num_qubits
        qs = list(range(n - 1, -1, -1)) if qubits is None else list(qubits)
        _validate_query(qs, n)
        probs = marginal_probs(self.state, n, qs)
        return {j: float(v) for j, v in enumerate(probs.tolist()) if v > 0.0}

    def counts(self, shots=1000, qubits=None, seed=None):
        n = self.num_qubits
        qs = list(range(n - 1, -1, -1)) if qubits is None else list(qubits)
        _validate_query(qs, n)
        seed = secrets.randbits(64) if seed is None else seed
        return sample_counts(self.state, n, shots, seed, qs)

    def fidelity(self, other):
        other = np.ascontiguousarray(other, dtype=np.complex128)
        if other.shape[0] != self.state.shape[0]:
            return 0.0
        return float(lib().orc_fidelity(_ptr(self.state), _ptr(other), other.shape[0]))


class OracleSimulator:
    """StatevectorSimulator restated on the CPU (simulator.rs:214-372)."""

    def __init__(self, seed=None, profile=False, *, max_memory_mb=1024, max_parallel_shots=None,
                 sample_terminal=True, threads=None):
        budget = max_memory_mb * 1024 * 1024
        if budget <= 0 or budget > ISIZE_MAX:
            raise ValueError("max_memory_mb must be positive and representable in bytes")
        if max_parallel_shots == 0:
            raise ValueError("max_parallel_shots must be positive or None")
        self.seed = seed
        self.budget = budget
        self.max_parallel_shots = max_parallel_shots
        self.sample_terminal = sample_terminal
        self.threads = threads

    def read(self, circuit):
        text = circuit if isinstance(circuit, str) else circuit.model_dump_json()
        c = parse_circuit(text)
        validate_circuit(c)
        return c

    def _seed(self):
        return self.seed if self.seed is not None else secrets.randbits(64)

    def simulate_shots_full(self, circuit, shots=1000):
        c = self.read(circuit)
        ops = compile_ops(c["instructions"])
        return run_shots(ops, num_qubits(c), num_cbits(c), shots, self._seed(), self.budget,
                         self.max_parallel_shots, self.sample_terminal, self.threads)

    def simulate_shots(self, circuit, shots=1000):
        return self.simulate_shots_full(circuit, shots)["counts"]

    def simulate(self, circuit):
        c = self.read(circuit)
        n, ncb = num_qubits(c), num_cbits(c)
        _, nbytes = state_layout(n)
        check_budget(nbytes + ncb, self.budget)
        ops = compile_ops(c["instructions"])
        state = zero_state(n)
        cbits = [0] * ncb
        execute(ops, state, n, cbits, ChaCha8Stream(self._seed()), True)
        return OracleResult(state, n, cbits)


def circuit_ops(circuit_json):
    """Parse, validate and compile a transport JSON string; returns (n, ncb, ops)."""
    c = parse_circuit(circuit_json)
    validate_circuit(c)
    return num_qubits(c), num_cbits(c), compile_ops(c["instructions"])


if __name__ == "__main__":  # pragma: no cover
    build()
    print("oracle threads:", lib().orc_num_threads(), "pid", os.getpid())

"""OpenQASM 2 to the dqsim transport, with a parser of this package's own.

The reference imports OpenQASM 2 through Qiskit (python/dqsim/qasm.py:173-221:
`load_qasm` parses with qiskit.qasm2, `from_qiskit` lowers the parsed circuit).
Qiskit is optional there and absent here, so `load_qasm` reads the source
itself and produces the same transport (`ImportedCircuit.model_dump_json()`,
the instruction schema of src/types.rs): registers laid out in declaration
order, every qelib1 / Qiskit-legacy standard gate kept as its own transport
kind (the transport has a kind for each, three- and four-qubit ones included),
user `gate` definitions expanded by their bodies, `measure`, `reset`,
`barrier` and register-broadcast operands, `if (creg == value)` conditions,
and parameter expressions (pi, + - * / ^, unary minus, sin cos tan exp ln
sqrt).  `from_qiskit` needs Qiskit and raises ImportError without it, as the
reference does.
"""

from __future__ import annotations

import hashlib
import json
import math
import re
from dataclasses import dataclass
from pathlib import Path


class QASMImportError(ValueError):
    """A source cannot be faithfully represented by the supported transport."""


@dataclass
class ImportedCircuit:
    data: dict
    metadata: dict

    def model_dump_json(self):
        return json.dumps(self.data, separators=(",", ":"), allow_nan=False)

    @property
    def num_qubits(self):
        return sum(reg["size"] for reg in self.data["qregs"].values())

    @property
    def num_cbits(self):
        return sum(reg["size"] for reg in self.data["cregs"].values())


def from_qiskit(circuit, *, max_instructions=250_000):
    """Lowering of a Qiskit circuit: needs Qiskit, which this environment does not provide."""
    try:
        import qiskit  # noqa: F401
    except ImportError as exc:
        raise ImportError('OpenQASM import from Qiskit circuits requires qiskit; load_qasm parses OpenQASM 2 '
                          'source without it') from exc
    raise NotImplementedError("lowering Qiskit circuit objects is not provided; export them with "
                              "qiskit.qasm2.dumps and use load_qasm")


# Transport operand and parameter names of each standard gate (src/types.rs:60-265).
_ONE = ("qubit",)
_TWO = ("control", "target")
_PAIR = ("a", "b")
STANDARD = {
    **{g: (_ONE, ()) for g in ("id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg")},
    "u3": (_ONE, ("theta", "phi", "lam")), "u": (_ONE, ("theta", "phi", "lam")), "u2": (_ONE, ("phi", "lam")),
    "u1": (_ONE, ("lam",)), "p": (_ONE, ("lam",)), "rx": (_ONE, ("theta",)), "ry": (_ONE, ("theta",)),
    "rz": (_ONE, ("phi",)),
    **{g: (_TWO, ()) for g in ("cx", "cz", "cy", "ch", "csx")},
    "crx": (_TWO, ("theta",)), "cry": (_TWO, ("theta",)), "crz": (_TWO, ("lam",)), "cu1": (_TWO, ("lam",)),
    "cp": (_TWO, ("lam",)), "cu3": (_TWO, ("theta", "phi", "lam")), "cu": (_TWO, ("theta", "phi", "lam", "gamma")),
    "swap": (_PAIR, ()), "rxx": (_PAIR, ("theta",)), "rzz": (_PAIR, ("theta",)),
    "ccx": (("control1", "control2", "target"), ()), "cswap": (("control", "target1", "target2"), ()),
    "rccx": (("control1", "control2", "target"), ()),
    "rc3x": (("control1", "control2", "control3", "target"), ()),
    "c3x": (("control1", "control2", "control3", "target"), ()),
    "c3sqrtx": (("control1", "control2", "control3", "target"), ()),
    "c4x": (("control1", "control2", "control3", "control4", "target"), ()),
}
# OpenQASM 2 built-ins and the idle gate (whose duration the transport does not keep).
_ALIASES = {"U": "u", "CX": "cx"}

_TOKEN = re.compile(r"""
    (?P<ws>\s+|//[^\n]*|/\*.*?\*/)
  | (?P<real>(?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)
  | (?P<int>\d+)
  | (?P<string>"[^"\n]*")
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>->|==|[;,()\[\]{}+\-*/^])
""", re.S | re.X)
_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log, "sqrt": math.sqrt}


def _tokens(text, where):
    out, pos, line = [], 0, 1
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m:
            raise QASMImportError(f"{where}:{line}: unexpected character {text[pos]!r}")
        kind = m.lastgroup
        if kind != "ws":
            out.append((kind, m.group(), line))
        line += m.group().count("\n")
        pos = m.end()
    out.append(("eof", "", line))
    return out


class _Parser:
    def __init__(self, tokens, where):
        self.t, self.i, self.where = tokens, 0, where

    def peek(self, k=0):
        return self.t[self.i + k]

    def error(self, msg):
        raise QASMImportError(f"{self.where}:{self.peek()[2]}: {msg}")

    def take(self, value=None, kind=None):
        tok = self.t[self.i]
        if (value is not None and tok[1] != value) or (kind is not None and tok[0] != kind):
            self.error(f"expected {value or kind}, found {tok[1] or 'end of input'!r}")
        self.i += 1
        return tok

    def accept(self, value):
        if self.t[self.i][1] == value and self.t[self.i][0] in ("op", "id"):
            self.i += 1
            return True
        return False

    # expressions: sum of terms; ^ binds tightest (right-associative), then unary minus
    def expr(self, env):
        v = self.term(env)
        while self.peek()[1] in ("+", "-"):
            v = v + self.term(env) if self.take()[1] == "+" else v - self.term(env)
        return v

    def term(self, env):
        v = self.unary(env)
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            rhs = self.unary(env)
            if op == "*":
                v *= rhs
            elif rhs == 0:
                self.error("division by zero")
            else:
                v /= rhs
        return v

    def unary(self, env):
        if self.accept("-"):
            return -self.unary(env)
        if self.accept("+"):
            return self.unary(env)
        return self.power(env)

    def power(self, env):
        base = self.atom(env)
        if self.accept("^"):
            return base ** self.unary(env)
        return base

    def atom(self, env):
        kind, text, _ = self.peek()
        if kind in ("real", "int"):
            self.i += 1
            return float(text)
        if kind == "id":
            self.i += 1
            if text == "pi":
                return math.pi
            if text in _FUNCS:
                self.take("(")
                v = self.expr(env)
                self.take(")")
                try:
                    return _FUNCS[text](v)
                except (ValueError, OverflowError):
                    self.error(f"{text}({v}) is undefined")
            if text in env:
                return env[text]
            self.error(f"unknown parameter {text!r}")
        if self.accept("("):
            v = self.expr(env)
            self.take(")")
            return v
        self.error(f"expected an expression, found {text or 'end of input'!r}")


class _Program:
    def __init__(self, include_path, max_source_bytes, max_instructions):
        self.qregs, self.cregs = {}, {}
        self.nq = self.nc = 0
        self.gates = {}  # user gate name -> (params, args, body tokens) or None for opaque
        self.out = []
        self.include_path = list(include_path)
        self.max_source_bytes = max_source_bytes
        self.max_instructions = max_instructions
        self.source_bytes = 0
        self.includes = []

    def emit(self, item):
        if len(self.out) >= self.max_instructions:
            raise QASMImportError(f"Expanded circuit exceeds {self.max_instructions} instructions")
        self.out.append(item)

    def run(self, text, where, directory, depth=0):
        if depth > 64:
            raise QASMImportError("Include nesting exceeds 64 levels")
        self.source_bytes += len(text.encode("utf-8"))
        if self.source_bytes > self.max_source_bytes:
            raise QASMImportError(f"Source/includes exceed {self.max_source_bytes} bytes")
        p = _Parser(_tokens(text, where), where)
        if depth == 0:
            p.take("OPENQASM")
            version = p.take()[1]
            if version not in ("2.0", "2"):
                p.error(f"only OpenQASM 2.0 is supported, not {version}")
            p.take(";")
        while p.peek()[0] != "eof":
            self.statement(p, directory, depth)

    def statement(self, p, directory, depth):
        kind, word, _ = p.peek()
        if word == "include":
            p.take()
            name = p.take(kind="string")[1][1:-1]
            p.take(";")
            if name == "qelib1.inc":
                return  # the standard gates are built in
            search = [directory] + self.include_path
            found = next((Path(d) / name for d in search if (Path(d) / name).is_file()), None)
            if found is None:
                p.error(f"Include not found: {name}")
            raw = found.read_bytes()
            self.includes.append({"path": str(found.resolve()), "sha256": hashlib.sha256(raw).hexdigest()})
            self.run(raw.decode("utf-8"), found.name, found.parent, depth + 1)
        elif word in ("qreg", "creg"):
            p.take()
            name = p.take(kind="id")[1]
            p.take("[")
            size = int(p.take(kind="int")[1])
            p.take("]")
            p.take(";")
            if name in self.qregs or name in self.cregs:
                p.error(f"register {name!r} is declared twice")
            if size < 1:
                p.error("registers hold at least one bit")
            if word == "qreg":
                self.qregs[name] = {"name": name, "base": self.nq, "size": size}
                self.nq += size
            else:
                self.cregs[name] = {"name": name, "base": self.nc, "size": size}
                self.nc += size
        elif word in ("gate", "opaque"):
            p.take()
            name = p.take(kind="id")[1]
            params = []
            if p.accept("("):
                if not p.accept(")"):
                    params.append(p.take(kind="id")[1])
                    while p.accept(","):
                        params.append(p.take(kind="id")[1])
                    p.take(")")
            args = [p.take(kind="id")[1]]
            while p.accept(","):
                args.append(p.take(kind="id")[1])
            if len(set(args)) != len(args) or len(set(params)) != len(params):
                p.error(f"gate {name!r} repeats a parameter or argument name")
            if word == "opaque":
                p.take(";")
                self.gates[name] = None
                return
            p.take("{")
            start, level = p.i, 1
            while level:
                tok = p.take()
                if tok[0] == "eof":
                    p.error(f"gate {name!r} has no closing brace")
                level += {"{": 1, "}": -1}.get(tok[1], 0) if tok[0] == "op" else 0
            self.gates[name] = (params, args, p.t[start:p.i - 1] + [("eof", "", p.t[p.i - 1][2])])
        elif word == "if":
            p.take()
            p.take("(")
            creg = p.take(kind="id")[1]
            p.take("==")
            value = int(p.take(kind="int")[1])
            p.take(")")
            if creg not in self.cregs:
                p.error(f"unknown classical register {creg!r}")
            reg = self.cregs[creg]
            if reg["size"] > 64 or value >= (1 << reg["size"]):
                p.error("condition value exceeds the register width")
            cond = {"creg_base": reg["base"], "creg_size": reg["size"], "creg_value": value}
            before = len(self.out)
            self.quantum_op(p)
            self.out[before:] = [{"kind": "conditional", "condition": dict(cond), "op": op} for op in self.out[before:]]
        else:
            self.quantum_op(p)

    def operand(self, p, regs, what):
        name = p.take(kind="id")[1]
        if name not in regs:
            p.error(f"unknown {what} register {name!r}")
        reg = regs[name]
        if p.accept("["):
            idx = int(p.take(kind="int")[1])
            p.take("]")
            if idx >= reg["size"]:
                p.error(f"index {idx} is outside register {name!r}")
            return [reg["base"] + idx]
        return [reg["base"] + k for k in range(reg["size"])]

    @staticmethod
    def broadcast(p, operands):
        sizes = {len(o) for o in operands if len(o) > 1}
        if len(sizes) > 1:
            p.error("register operands of different sizes")
        width = sizes.pop() if sizes else 1
        return [[o[k] if len(o) > 1 else o[0] for o in operands] for k in range(width)]

    def quantum_op(self, p):
        word = p.take(kind="id")[1]
        if word == "measure":
            q = self.operand(p, self.qregs, "quantum")
            p.take("->")
            c = self.operand(p, self.cregs, "classical")
            p.take(";")
            if len(q) != len(c):
                p.error("measure needs operands of the same size")
            for qq, cc in zip(q, c):
                self.emit({"kind": "measure", "qubit": qq, "cbit": cc})
            return
        if word == "reset":
            q = self.operand(p, self.qregs, "quantum")
            p.take(";")
            for qq in q:
                self.emit({"kind": "reset", "qubit": qq})
            return
        if word == "barrier":
            self.operand(p, self.qregs, "quantum")
            while p.accept(","):
                self.operand(p, self.qregs, "quantum")
            p.take(";")
            self.emit({"kind": "barrier"})  # the transport's barrier is global
            return
        params = []
        if p.accept("("):
            if not p.accept(")"):
                params.append(p.expr({}))
                while p.accept(","):
                    params.append(p.expr({}))
                p.take(")")
        operands = [self.operand(p, self.qregs, "quantum")]
        while p.accept(","):
            operands.append(self.operand(p, self.qregs, "quantum"))
        p.take(";")
        for qubits in self.broadcast(p, operands):
            self.call(p, word, params, qubits, 0)

    def call(self, p, name, params, qubits, depth):
        if depth > 64:
            p.error("gate expansion exceeds 64 levels")
        if len(set(qubits)) != len(qubits):
            p.error(f"{name} repeats a qubit")
        if any(not math.isfinite(v) for v in params):
            p.error(f"nonfinite parameter in {name}")
        if name in self.gates:
            definition = self.gates[name]
            if definition is None:
                p.error(f"Unsupported opaque operation: {name}")
            names, args, body = definition
            if len(params) != len(names) or len(qubits) != len(args):
                p.error(f"{name} takes {len(names)} parameters and {len(args)} qubits")
            self.expand(body, dict(zip(names, params)), dict(zip(args, qubits)), depth, p.where)
            return
        std = _ALIASES.get(name, name)
        if std == "u0":  # an idle step: its duration parameter is not kept
            if len(qubits) != 1 or len(params) > 1:
                p.error("u0 takes one qubit")
            self.emit({"kind": "u0", "qubit": qubits[0]})
            return
        if std not in STANDARD:
            p.error(f"unknown gate {name!r}")
        operands, fields = STANDARD[std]
        if len(qubits) != len(operands) or len(params) != len(fields):
            p.error(f"{name} takes {len(fields)} parameters and {len(operands)} qubits")
        self.emit({"kind": std, **dict(zip(operands, qubits)), **dict(zip(fields, params))})

    def expand(self, body, env, wires, depth, where):
        p = _Parser(body, where)
        while p.peek()[0] != "eof":
            name = p.take(kind="id")[1]
            if name == "barrier":
                p.take(kind="id")
                while p.accept(","):
                    p.take(kind="id")
                p.take(";")
                self.emit({"kind": "barrier"})
                continue
            params = []
            if p.accept("("):
                if not p.accept(")"):
                    params.append(p.expr(env))
                    while p.accept(","):
                        params.append(p.expr(env))
                    p.take(")")
            qubits = []
            arg = p.take(kind="id")[1]
            while True:
                if arg not in wires:
                    p.error(f"unknown gate argument {arg!r}")
                qubits.append(wires[arg])
                if not p.accept(","):
                    break
                arg = p.take(kind="id")[1]
            p.take(";")
            self.call(p, name, params, qubits, depth + 1)


def parse_qasm(source, *, name="<source>", include_path=(), directory=".", max_source_bytes=8 * 1024 ** 2,
               max_instructions=250_000) -> ImportedCircuit:
    """OpenQASM 2 source text to the transport (includes resolve from `directory`, then `include_path`)."""
    if not isinstance(max_source_bytes, int) or max_source_bytes < 1:
        raise ValueError("max_source_bytes must be a positive integer")
    if not isinstance(max_instructions, int) or max_instructions < 1:
        raise ValueError("max_instructions must be a positive integer")
    prog = _Program([str(Path(d)) for d in include_path], max_source_bytes, max_instructions)
    prog.run(source, name, Path(directory))
    data = {"qregs": prog.qregs, "cregs": prog.cregs, "instructions": prog.out}
    meta = {"normalization": "standard-gates-native-v1", "parser": "dqsim-b200.qasm2",
            "source_sha256": hashlib.sha256(source.encode("utf-8")).hexdigest(), "includes": prog.includes}
    return ImportedCircuit(data, meta)


def load_qasm(path, *, include_path=(), legacy_gates=True, max_source_bytes=8 * 1024 ** 2,
              max_instructions=250_000) -> ImportedCircuit:
    """Read an OpenQASM 2 file and lower it to the transport (python/dqsim/qasm.py:173-221).

    With legacy_gates the gates Qiskit adds to qelib1.inc (rccx, rc3x, c3x, c3sqrtx, c4x, cu, p, cp, sx, sxdg,
    csx, rxx) are known without a definition; without it a circuit that uses one and does not define it is
    rejected.  A `gate` definition of the same name in the source always takes precedence."""
    path = Path(path).resolve()
    try:
        raw = path.read_bytes()
        source = raw.decode("utf-8")
    except (OSError, UnicodeError) as exc:
        raise QASMImportError(f"{path.name}: {exc}") from exc
    if len(raw) > max_source_bytes:
        raise QASMImportError(f"Source/includes exceed {max_source_bytes} bytes")
    imported = parse_qasm(source, name=path.name, include_path=include_path, directory=path.parent,
                          max_source_bytes=max_source_bytes, max_instructions=max_instructions)
    if not legacy_gates:
        legacy = {"rccx", "rc3x", "c3x", "c3sqrtx", "c4x", "cu", "p", "cp", "sx", "sxdg", "csx", "rxx"}

        def used(item):
            return used(item["op"]) if item["kind"] == "conditional" else item["kind"]
        bad = sorted({used(i) for i in imported.data["instructions"]} & legacy)
        if bad:
            raise QASMImportError(f"{path.name}: gates outside qelib1.inc without legacy_gates: {', '.join(bad)}")
    imported.metadata.update(source=str(path), legacy_gates=legacy_gates)
    return imported

"""OpenQASM 2 import (dqsim.qasm) without Qiskit.

The reference imports OpenQASM 2 through Qiskit (python/dqsim/qasm.py:173-221)
and its Qiskit tests (tests/test_statevector.py:404-486) skip here.  These
tests pin the package's own parser: the transport it produces for standard
gates, user gate definitions, broadcasting, measurement, conditions and
includes; the errors it raises; and that a circuit read from QASM simulates
exactly like the same circuit written in the transport (CPU oracle, and the
device engine in the GPU test).
"""

import json

import numpy as np
import pytest

from helpers import Circuit, inst
from oracle import oracle as o

import dqsim
from dqsim import QASMImportError, load_qasm, parse_qasm

HEAD = 'OPENQASM 2.0;\ninclude "qelib1.inc";\n'


def test_standard_gates_definitions_broadcast_measure_and_conditions():
    src = HEAD + """
qreg q[3]; creg c[3];
gate bell(t) a, b { h a; cx a, b; rz(t/2) b; }
h q;
bell(pi) q[0], q[1];
ccx q[0], q[1], q[2];
U(0.1, 0.2, -pi^2) q[2];
barrier q;
measure q -> c;
if (c == 5) x q[1];
"""
    c = parse_qasm(src)
    assert c.num_qubits == 3 and c.num_cbits == 3
    assert json.loads(c.model_dump_json()) == {
        "qregs": {"q": {"name": "q", "base": 0, "size": 3}},
        "cregs": {"c": {"name": "c", "base": 0, "size": 3}},
        "instructions": [
            {"kind": "h", "qubit": 0}, {"kind": "h", "qubit": 1}, {"kind": "h", "qubit": 2},
            {"kind": "h", "qubit": 0}, {"kind": "cx", "control": 0, "target": 1},
            {"kind": "rz", "qubit": 1, "phi": np.pi / 2},
            {"kind": "ccx", "control1": 0, "control2": 1, "target": 2},
            {"kind": "u", "qubit": 2, "theta": 0.1, "phi": 0.2, "lam": -np.pi ** 2},
            {"kind": "barrier"},
            {"kind": "measure", "qubit": 0, "cbit": 0}, {"kind": "measure", "qubit": 1, "cbit": 1},
            {"kind": "measure", "qubit": 2, "cbit": 2},
            {"kind": "conditional", "condition": {"creg_base": 0, "creg_size": 3, "creg_value": 5},
             "op": {"kind": "x", "qubit": 1}},
        ]}


def test_registers_lay_out_in_declaration_order_and_expressions_evaluate():
    src = HEAD + """
qreg a[2]; qreg b[3]; creg m[2]; creg n[1];
cu3(sin(pi/2), cos(0)*2, sqrt(4)-ln(exp(1))) a[1], b[2];
rzz(2^3^2 / 256) a[0], b;
measure b[1] -> n[0];
"""
    c = parse_qasm(src)
    d = c.data
    assert d["qregs"]["b"] == {"name": "b", "base": 2, "size": 3}
    assert d["cregs"]["n"] == {"name": "n", "base": 2, "size": 1}
    ins = d["instructions"]
    assert ins[0] == {"kind": "cu3", "control": 1, "target": 4, "theta": 1.0, "phi": 2.0, "lam": 1.0}
    assert [x["b"] for x in ins[1:4]] == [2, 3, 4] and all(x["a"] == 0 and x["theta"] == 2.0 for x in ins[1:4])
    assert ins[4] == {"kind": "measure", "qubit": 3, "cbit": 2}


def test_qasm_circuit_simulates_like_the_transport_circuit():
    src = HEAD + """
qreg q[4]; creg c[4];
gate layer(a, b) x0, x1 { ry(a) x0; rz(b) x1; cz x0, x1; }
layer(0.3, 1.1) q[0], q[1];
layer(-0.7, 0.2) q[2], q[3];
cswap q[0], q[1], q[3];
rc3x q[3], q[2], q[1], q[0];
cp(pi/5) q[1], q[2];
"""
    got = o.OracleSimulator(seed=1).simulate(parse_qasm(src)).statevector
    ins = [inst("ry", qubit=0, theta=0.3), inst("rz", qubit=1, phi=1.1), inst("cz", control=0, target=1),
           inst("ry", qubit=2, theta=-0.7), inst("rz", qubit=3, phi=0.2), inst("cz", control=2, target=3),
           inst("cswap", control=0, target1=1, target2=3),
           inst("rc3x", control1=3, control2=2, control3=1, target=0),
           inst("cp", control=1, target=2, lam=np.pi / 5)]
    want = o.OracleSimulator(seed=1).simulate(Circuit(4, ins)).statevector
    assert np.array_equal(got, want)


def test_includes_resolve_from_the_file_and_the_include_path(tmp_path):
    lib = tmp_path / "lib"
    lib.mkdir()
    (lib / "mine.inc").write_text("gate twice a { x a; x a; }\n")
    (tmp_path / "local.inc").write_text('include "mine.inc";\ngate flip a { x a; }\n')
    main = tmp_path / "main.qasm"
    main.write_text(HEAD + 'include "local.inc";\nqreg q[1];\nflip q[0];\ntwice q[0];\n')
    c = load_qasm(main, include_path=[lib])
    assert [i["kind"] for i in c.data["instructions"]] == ["x", "x", "x"]
    assert [x["path"] for x in c.metadata["includes"]] == [str((tmp_path / "local.inc").resolve()),
                                                         str((lib / "mine.inc").resolve())]
    assert c.metadata["source"] == str(main.resolve())
    with pytest.raises(QASMImportError, match="Include not found"):
        load_qasm(main)


def test_legacy_gates_flag(tmp_path):
    f = tmp_path / "c.qasm"
    f.write_text(HEAD + "qreg q[3];\nrccx q[0], q[1], q[2];\n")
    assert load_qasm(f).data["instructions"][0]["kind"] == "rccx"
    with pytest.raises(QASMImportError, match="legacy"):
        load_qasm(f, legacy_gates=False)
    f.write_text(HEAD + "qreg q[3];\ngate rccx a, b, c { ccx a, b, c; }\nrccx q[0], q[1], q[2];\n")
    assert load_qasm(f, legacy_gates=False).data["instructions"][0]["kind"] == "ccx"


@pytest.mark.parametrize("body, match", [
    ("qreg q[2];\nfoo q[0];", "unknown gate"),
    ("qreg q[2];\nopaque magic a;\nmagic q[0];", "opaque"),
    ("qreg q[2]; qreg r[3];\ncx q, r;", "different sizes"),
    ("qreg q[2];\nx q[2];", "outside register"),
    ("qreg q[2];\ncx q[0], q[0];", "repeats a qubit"),
    ("qreg q[2]; qreg q[3];", "declared twice"),
    ("qreg q[1];\nrx(ln(0)) q[0];", "undefined"),
    ("qreg q[1];\nrx(1/0) q[0];", "division by zero"),
    ("qreg q[1]; creg c[1];\nif (c == 2) x q[0];", "exceeds"),
    ("qreg q[1];\nu3(1, 2) q[0];", "takes 3 parameters"),
    ("qreg q[1];\nh q[0]", "expected ;"),
])
def test_invalid_sources_raise(body, match):
    with pytest.raises(QASMImportError, match=match):
        parse_qasm(HEAD + body)


def test_header_limits_and_qiskit_lowering():
    with pytest.raises(QASMImportError):
        parse_qasm("qreg q[1];")
    with pytest.raises(QASMImportError, match="only OpenQASM 2.0"):
        parse_qasm("OPENQASM 3.0;")
    with pytest.raises(QASMImportError, match="exceeds 5 instructions"):
        parse_qasm(HEAD + "qreg q[6];\nh q;", max_instructions=5)
    with pytest.raises(ImportError):
        dqsim.from_qiskit(object())


@pytest.mark.gpu
def test_device_engine_runs_an_imported_circuit():
    src = HEAD + """
qreg q[13]; creg c[13];
gate mix(t) a, b { ry(t) a; cx a, b; u2(t, -t) b; }
h q;
mix(0.4) q[0], q[12];
mix(1.3) q[5], q[6];
c3sqrtx q[1], q[2], q[3], q[4];
"""
    c = parse_qasm(src)
    got = dqsim.StatevectorSimulator(seed=3).simulate(c).statevector
    want = o.OracleSimulator(seed=3).simulate(c).statevector
    assert np.max(np.abs(got - want)) <= 1e-12

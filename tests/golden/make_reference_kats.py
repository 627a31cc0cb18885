"""Writes reference_kats.json: the known-answer tables of the reference's own tests.

The reference (dqsim 0.1.2) is Rust and cannot be built here, so its outputs
cannot be regenerated; these tables transcribe the expectations its tests
assert, with the file:line each one comes from.  They pin the CPU oracle
(tests/test_oracle_kats.py) and the product's host validation
(tests/test_host_abi.py).  Run: python tests/golden/make_reference_kats.py
"""

import json
from pathlib import Path

USIZE_MAX = (1 << 64) - 1
U64_MAX = (1 << 64) - 1


def inst(kind, **f):
    return {"kind": kind, **f}


def cond(base, size, value, op):
    return inst("conditional", condition={"creg_base": base, "creg_size": size, "creg_value": value}, op=op)


def gen(name, qubits, params):
    return inst("gate", name=name, qubits=qubits, params=params)


def regs(*specs):
    return {name: {"name": name, "base": base, "size": size} for name, base, size in specs}


KATS = {
    "source": "dqsim 0.1.2 test suites; see per-entry `ref`",
    # src/engine.rs:689-705: amplitudes sqrt(i/36), i = 1..8
    "marginal_probs": [
        {"ref": "src/engine.rs:695", "qubits": [0, 2], "expected_x36": [4.0, 12.0, 6.0, 14.0]},
        {"ref": "src/engine.rs:696", "qubits": [2, 0], "expected_x36": [4.0, 6.0, 12.0, 14.0]},
        {"ref": "src/engine.rs:697", "qubits": [], "expected_x36": [36.0]},
        {"ref": "src/engine.rs:698", "qubits": [2, 1, 0], "expected_x36": [float(i) for i in range(1, 9)]},
    ],
    "validation_accept": [
        {"ref": "statevector/validation.rs:56-73",
         "instructions": [inst("h", qubit=0), inst("cx", control=0, target=2), inst("measure", qubit=2, cbit=1),
                          cond(0, 3, 2, cond(1, 1, 1, inst("reset", qubit=0)))]},
        {"ref": "statevector/validation.rs:129", "instructions": [gen("remote_cu1", [0, 1], [0.4])]},
        {"ref": "statevector/validation.rs:130", "instructions": [gen("remote_rzz", [0, 1], [0.4])]},
        {"ref": "statevector/validation.rs:131", "instructions": [gen("REMOTE_CX", [0, 2], [])]},
        {"ref": "statevector/validation.rs:132", "instructions": [gen("remote_barrier", [0, 1, 2], [])]},
        {"ref": "statevector/validation.rs:191-198", "cregs": regs(("c", 0, 64)),
         "instructions": [cond(0, 64, U64_MAX, inst("x", qubit=0))]},
    ],
    "validation_reject": [
        {"ref": "statevector/validation.rs:78-81", "instructions": [inst("cx", control=0, target=3)]},
        {"ref": "statevector/validation.rs:82-85", "instructions": [inst("cx", control=1, target=1)]},
        {"ref": "statevector/validation.rs:86", "instructions": [inst("id", qubit=3)]},
        {"ref": "statevector/validation.rs:87", "instructions": [inst("measure", qubit=0, cbit=3)]},
        {"ref": "statevector/validation.rs:88", "instructions": [cond(0, 1, 1, inst("x", qubit=99))]},
        {"ref": "statevector/validation.rs:92-98", "qregs": regs(("a", 0, 1), ("b", 2, 1)),
         "instructions": [inst("x", qubit=1)]},
        {"ref": "statevector/validation.rs:99-105", "qregs": regs(("q", 0, 12)),
         "instructions": [inst("cx", control=0, target=12)]},
        {"ref": "statevector/validation.rs:111", "qregs": regs(("a", USIZE_MAX, 1)), "instructions": []},
        {"ref": "statevector/validation.rs:112", "qregs": regs(("a", 0, 2), ("b", 1, 2)), "instructions": []},
        {"ref": "statevector/validation.rs:113", "qregs": regs(("a", 0, 64)), "instructions": []},
        {"ref": "statevector/validation.rs:119-123", "cregs": regs(("c", 0, 3), ("overlap", 1, 1)),
         "instructions": []},
        {"ref": "statevector/validation.rs:137", "instructions": [gen("remote_cu1", [0, 1], [])]},
        {"ref": "statevector/validation.rs:138", "instructions": [gen("remote_cx", [0], [])]},
        {"ref": "statevector/validation.rs:139", "instructions": [gen("remote_epr", [0, 1, 2], [])]},
        {"ref": "statevector/validation.rs:140", "instructions": [gen("remote_cz", [0, 1], [0.2])]},
        {"ref": "statevector/validation.rs:141", "instructions": [gen("circuit-123", [0], [])]},
        {"ref": "statevector/validation.rs:142", "instructions": [gen("remote_barrier", [1, 1], [])]},
        {"ref": "statevector/validation.rs:143-145", "instructions": [inst("classical", name="opaque")]},
        {"ref": "statevector/validation.rs:154-159",
         "instructions": [inst("u3", qubit=0, theta=0.0, phi=float("nan"), lam=0.0)]},
        {"ref": "statevector/validation.rs:160-167",
         "instructions": [inst("cu", control=0, target=1, theta=0.0, phi=0.0, lam=0.0, gamma=float("inf"))]},
        {"ref": "statevector/validation.rs:168", "instructions": [gen("remote_rzz", [0, 1], [float("-inf")])]},
        {"ref": "statevector/validation.rs:169-173",
         "instructions": [inst("u2", qubit=0, phi=1.7976931348623157e308, lam=1.7976931348623157e308)]},
        {"ref": "statevector/validation.rs:182", "instructions": [cond(0, 0, 0, inst("x", qubit=0))]},
        {"ref": "statevector/validation.rs:183", "instructions": [cond(0, 65, 0, inst("x", qubit=0))]},
        {"ref": "statevector/validation.rs:184", "instructions": [cond(0, 1, 2, inst("x", qubit=0))]},
        {"ref": "statevector/validation.rs:185", "instructions": [cond(2, 2, 0, inst("x", qubit=0))]},
        {"ref": "statevector/validation.rs:186", "instructions": [cond(USIZE_MAX, 2, 0, inst("x", qubit=0))]},
    ],
    # tests/test_statevector.py:215-232 (ValueError before execution)
    "api_invalid": [
        {"n": 12, "cbits": 0, "instructions": [inst("cx", control=0, target=12)]},
        {"n": 12, "cbits": 0, "instructions": [inst("x", qubit=12)]},
        {"n": 2, "cbits": 0, "instructions": [inst("cx", control=1, target=1)]},
        {"n": 3, "cbits": 0, "instructions": [inst("ccx", control1=0, control2=0, target=2)]},
        {"n": 2, "cbits": 2, "instructions": [inst("measure", qubit=0, cbit=2)]},
        {"n": 1, "cbits": 1, "instructions": [cond(0, 1, 1, inst("x", qubit=1))]},
        {"n": 1, "cbits": 1, "instructions": [cond(1, 1, 0, inst("x", qubit=0))]},
        {"n": 2, "cbits": 0, "instructions": [gen("remote_cx", [0], [])]},
        {"n": 2, "cbits": 0, "instructions": [gen("remote_cu1", [0, 1], [])]},
    ],
    # tests/test_statevector.py:234-248 (ValueError or NotImplementedError)
    "api_unsupported": [
        gen("circuit-123", [0], []),
        gen("unknown", [0], []),
        inst("classical", name="unsupported_classical_operation"),
    ],
}

if __name__ == "__main__":
    out = Path(__file__).with_name("reference_kats.json")
    out.write_text(json.dumps(KATS, indent=1) + "\n")
    print("wrote", out)

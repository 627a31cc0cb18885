"""Host-side checks of the product through its C ABI (no GPU needed).

* the library loads and exports every entry point include/dqsim_sv.h declares;
* parse + validation + 1q fusion give exactly the oracle's operation list
  (bit patterns of every matrix entry) on seeded random circuits of every gate;
* option, circuit and budget errors surface with the reference's exception
  classes before any device work.
"""

import ctypes
import json
import math
import re
import struct
from pathlib import Path

import numpy as np
import pytest

from helpers import Circuit, conditional, inst, random_circuit
from oracle import oracle as o

import dqsim
from dqsim import _core

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = json.loads((ROOT / "tests" / "golden" / "reference_kats.json").read_text())


def header_symbols():
    text = (ROOT / "include" / "dqsim_sv.h").read_text()
    return sorted(set(re.findall(r"DQ_API\s+[\w\s\*]+?\b(dq_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_core.library_path())
    syms = header_symbols()
    assert len(syms) >= 20
    for name in syms:
        assert hasattr(lib, name), name


def test_call_phase_count_matches_the_header():
    text = (ROOT / "include" / "dqsim_sv.h").read_text()
    declared = int(re.search(r"#define DQ_CALL_PHASES (\d+)", text).group(1))
    assert declared == len(_core.CALL_PHASES) == 12
    assert _core.CALL_PHASES[-2:] == ("table", "prefix_device")


def _bits(x):
    return "%016x" % struct.unpack("<Q", struct.pack("<d", x))[0]


def _oracle_dump(op):
    kind = op[0]
    if kind == "one":
        return {"op": "one", "target": op[1], "controls": [[q, int(v)] for q, v in op[3]],
                "m": [[_bits(v.real), _bits(v.imag)] for row in op[2] for v in row]}
    if kind == "x":
        return {"op": "x", "target": op[1], "controls": [[q, int(v)] for q, v in op[2]]}
    if kind == "swap":
        return {"op": "swap", "a": op[1], "b": op[2], "controls": [[q, int(v)] for q, v in op[3]]}
    if kind == "diag":
        return {"op": "diag", "qubits": list(op[1]), "values": [[_bits(v.real), _bits(v.imag)] for v in op[2]]}
    if kind == "dense":
        return {"op": "dense", "qubits": list(op[1]),
                "values": [[_bits(v.real), _bits(v.imag)] for row in op[2] for v in row]}
    if kind == "measure":
        return {"op": "measure", "qubit": op[1], "cbit": op[2]}
    if kind == "reset":
        return {"op": "reset", "qubit": op[1]}
    if kind == "cond":
        return {"op": "cond", "condition": list(op[1]), "inner": _oracle_dump(op[2])}
    if kind == "noop":
        return {"op": "noop"}
    raise AssertionError(kind)


@pytest.mark.parametrize("seed", range(12))
def test_compiled_operations_match_oracle_bit_for_bit(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 9))
    ins = random_circuit(seed, n, 60)
    # sprinkle measurements, resets and conditionals
    cb = 4
    extra = []
    for i, x in enumerate(ins):
        extra.append(x)
        if i % 17 == 5:
            extra.append(inst("measure", qubit=int(rng.integers(n)), cbit=int(rng.integers(cb))))
        if i % 23 == 7:
            extra.append(conditional(x, int(rng.integers(2)), base=int(rng.integers(cb)), size=1))
        if i % 29 == 11:
            extra.append(inst("reset", qubit=int(rng.integers(n))))
    text = Circuit(n, extra, cb).model_dump_json()
    got = _core.compile_dump(text)
    want = [_oracle_dump(op) for op in o.circuit_ops(text)[2]]
    assert got == want


def test_brickwork_fusion_counts():
    from helpers import brickwork

    text = brickwork(10, 6, seed=0).model_dump_json()
    got = _core.compile_dump(text)
    want = [_oracle_dump(op) for op in o.circuit_ops(text)[2]]
    assert got == want
    kinds = [g["op"] for g in got]
    assert kinds.count("measure") == 10


@pytest.mark.parametrize("case", GOLDEN["validation_accept"] + GOLDEN["validation_reject"])
def test_validation_tables_through_abi(case):
    qregs = case.get("qregs") or {"q": {"name": "q", "base": 0, "size": 3}}
    cregs = case.get("cregs") or {"c": {"name": "c", "base": 0, "size": 3}}
    text = json.dumps({"qregs": qregs, "cregs": cregs, "instructions": case["instructions"]})
    if case in GOLDEN["validation_accept"]:
        _core.compile_dump(text)
    else:
        with pytest.raises(ValueError):
            _core.compile_dump(text)


@pytest.mark.parametrize("case", GOLDEN["api_invalid"])
def test_invalid_circuits_raise_value_error_before_execution(case):
    c = Circuit(case["n"], case["instructions"], case["cbits"])
    s = dqsim.StatevectorSimulator(seed=1)
    for method in (s.simulate, s.simulate_shots):
        with pytest.raises(ValueError):
            method(c)


@pytest.mark.parametrize("op", GOLDEN["api_unsupported"])
def test_unsupported_operations_are_never_silently_ignored(op):
    s = dqsim.StatevectorSimulator(seed=1)
    for instruction in (op, conditional(op, 1)):
        c = Circuit(1, [instruction], cbits=1)
        for method in (s.simulate, s.simulate_shots):
            with pytest.raises((ValueError, NotImplementedError)):
                method(c)


def test_memory_budget_rejects_oversized_state_before_allocation():
    s = dqsim.StatevectorSimulator(max_memory_mb=1)
    for method in (s.simulate, s.simulate_shots):
        with pytest.raises((ValueError, MemoryError)):
            method(Circuit(20))


def test_invalid_options_and_large_classical_registers():
    for options in ({"max_memory_mb": 0}, {"max_parallel_shots": 0}):
        with pytest.raises(ValueError):
            dqsim.StatevectorSimulator(**options)
    with pytest.raises(TypeError):
        dqsim.simulate_monolithic(Circuit(1), nonexistent_option=True)
    c = Circuit(1, cbits=2_000_000)
    s = dqsim.StatevectorSimulator(max_memory_mb=1)
    for method in (s.simulate, s.simulate_shots):
        with pytest.raises(MemoryError):
            method(c)


def test_zero_shots_return_empty_without_a_device():
    s = dqsim.StatevectorSimulator(seed=30)
    assert s.simulate_shots(Circuit(40, [inst("h", qubit=0)], cbits=3), shots=0) == {}


def test_json_errors_are_value_errors():
    s = dqsim.StatevectorSimulator(seed=1)

    class Raw:
        def __init__(self, text):
            self.text = text

        def model_dump_json(self):
            return self.text

    bad = [
        "{", "[]", '{"qregs": {}}', '{"qregs": {}, "instructions": [{"kind": "nope"}]}',
        '{"qregs": {"q": {"name": "q", "base": 0, "size": 1.0}}, "instructions": []}',
        '{"qregs": {"q": {"name": "q", "base": -1, "size": 1}}, "instructions": []}',
        '{"qregs": {"q": {"name": "q", "base": 0, "size": 1}}, "instructions": [{"kind": "rx", "qubit": 0}]}',
        '{"qregs": {"q": {"name": "q", "base": 0, "size": 1}}, "instructions": [{"kind": "rx", "qubit": 0, "theta": NaN}]}',
        '{"qregs": {"q": {"name": "q", "base": 0, "size": 1}}, "instructions": []} x',
        '{"qregs": {"q": {"name": "q", "base": 0, "size": 99999999999999999999}}, "instructions": []}',
    ]
    for text in bad:
        with pytest.raises(ValueError):
            s.simulate(Raw(text))


def test_modes_and_other_backends():
    with pytest.raises(ValueError):
        dqsim.simulate_monolithic(Circuit(1), mode="nope")
    with pytest.raises(NotImplementedError):
        dqsim.simulate_monolithic(Circuit(1), mode="mps")
    with pytest.raises(NotImplementedError):
        dqsim.MpsSimulator()
    with pytest.raises(NotImplementedError):
        dqsim.simulate_distributed(None)


def test_profile_repr_format():
    class P:
        apply_one_qubit_calls, apply_one_qubit_time = 3, 0.001
        apply_n_qubit_calls, apply_n_qubit_time = 2, 0.002
        measure_qubit_calls, measure_qubit_time = 1, 0.0005
        total_time = 0.004

    text = repr(_core.SimulationProfile(P()))
    assert text.startswith("SimulationProfile (total: 4.00 ms)")
    assert "apply_one_qubit :    3 calls      1.00 ms  (25.0%)" in text

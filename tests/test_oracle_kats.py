"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates one reference test (file:line in the dqsim project) against
oracle/oracle.py, so the oracle used by the GPU parity tests is anchored to
what the reference asserts about itself.  No GPU needed.
"""

import ctypes
import json
import math
import struct

import numpy as np
import pytest

from helpers import Circuit, assert_distribution, conditional, inst
from oracle import oracle as o

GOLDEN = json.loads((__import__("pathlib").Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def engine_input(n):
    """src/engine.rs:515-524."""
    i = np.arange(1 << n, dtype=np.float64)
    s = np.sin(i + 0.25) + 1j * np.cos(i + 0.5)
    return (s / np.sqrt(np.sum(np.abs(s) ** 2))).astype(np.complex128)


def fourier(dim):
    """src/engine.rs:553-566."""
    r = np.arange(dim)
    return np.exp(2j * np.pi * np.outer(r, r) / dim) / math.sqrt(dim)


def dense_reference(state, matrix, qubits):
    """Independent out-of-place reference, src/engine.rs:535-551."""
    out = np.zeros_like(state)
    k = len(qubits)
    for basis in range(len(state)):
        row = 0
        for q in qubits:
            row = 2 * row + ((basis >> q) & 1)
        for col in range(1 << k):
            src = basis
            for pos, q in enumerate(qubits):
                src &= ~(1 << q)
                src |= ((col >> (k - 1 - pos)) & 1) << q
            out[basis] += matrix[row][col] * state[src]
    return out


def apply_dense(state, n, qubits, matrix, parallel):
    s = state.copy()
    qs = o._ints(qubits)
    u = o._cplx(np.asarray(matrix).reshape(-1))
    o.lib().orc_apply_dense(o._ptr(s), n, o._ptr(qs), len(qubits), o._ptr(u), 1 if parallel else 0)
    return s


def close(a, b, tol=1e-12):
    assert np.max(np.abs(a - b)) < tol


@pytest.mark.parametrize("n", [5, 12])
def test_dense_gates_match_reference_for_target_order_and_parallel(n):
    # src/engine.rs:568-590
    original = engine_input(n)
    for qs in ([0], [n - 1], [n - 1, 0], [0, 3, 1], [4, 2, 0, 3, 1], []):
        m = fourier(1 << len(qs))
        expected = dense_reference(original, m, qs)
        close(apply_dense(original, n, qs, m, False), expected)
        close(apply_dense(original, n, qs, m, True), expected)


@pytest.mark.parametrize("n", [4, 12])
def test_controlled_one_qubit_and_x_match_dense_reference(n):
    # src/engine.rs:592-639
    f = fourier(2)
    for target in (0, n - 1):
        control = n - 1 if target == 0 else 0
        for value in (False, True):
            for is_x in (False, True):
                m = np.zeros((4, 4), dtype=complex)
                for r in range(4):
                    for c in range(4):
                        if r // 2 != c // 2:
                            continue
                        if r // 2 == int(value):
                            m[r, c] = float(r % 2 != c % 2) if is_x else f[r % 2, c % 2]
                        else:
                            m[r, c] = float(r == c)
                original = engine_input(n)
                expected = dense_reference(original, m, [control, target])
                for parallel in (0, 1):
                    s = original.copy()
                    cq, cv = o._ints([control]), o._ints([int(value)])
                    u = o._cplx(f.reshape(-1))
                    o.lib().orc_apply_one_qubit(o._ptr(s), n, target, o._ptr(u), o._ptr(cq), o._ptr(cv), 1,
                                                int(is_x), parallel)
                    close(s, expected)


@pytest.mark.parametrize("n", [4, 12, 13])
def test_diagonal_and_controlled_swap_match_dense_reference(n):
    # src/engine.rs:641-687
    original = engine_input(n)
    for qs in ([0, n - 1], [n - 1, 0]):
        diag = np.exp(1j * 0.3 * np.arange(4))
        expected = dense_reference(original, np.diag(diag), qs)
        for parallel in (0, 1):
            s = original.copy()
            qa, d = o._ints(qs), o._cplx(diag)
            o.lib().orc_apply_diagonal(o._ptr(s), n, o._ptr(qa), 2, o._ptr(d), parallel)
            close(s, expected)
    for a, b in ((0, n - 1), (n - 1, 0), (n - 1, n - 2)):
        control = next(q for q in range(n) if q not in (a, b))
        for controls in ([], [(control, True)], [(control, False)]):
            qubits = [a, b] if not controls else [control, a, b]
            dim = 1 << len(qubits)
            m = np.zeros((dim, dim), dtype=complex)
            for src in range(dim):
                enabled = not controls or (src // 4 == int(controls[0][1]))
                dest = ((src & ~3) | ((src & 1) << 1) | ((src & 2) >> 1)) if enabled else src
                m[dest, src] = 1
            expected = dense_reference(original, m, qubits)
            for parallel in (0, 1):
                s = original.copy()
                cq, cv = o._ints([c for c, _ in controls]), o._ints([int(v) for _, v in controls])
                o.lib().orc_apply_swap(o._ptr(s), n, a, b, o._ptr(cq), o._ptr(cv), len(controls), parallel)
                close(s, expected)


def test_marginal_probabilities_kat():
    # src/engine.rs:689-705 (golden table in tests/golden/reference_kats.json)
    state = np.sqrt(np.arange(1, 9) / 36.0).astype(np.complex128)
    for case in GOLDEN["marginal_probs"]:
        actual = o.marginal_probs(state, 3, case["qubits"])
        np.testing.assert_allclose(actual, np.asarray(case["expected_x36"]) / 36.0, atol=1e-14, rtol=0)


def test_sampling_skips_zero_probability_at_zero_draw():
    # src/engine.rs:707-731: StepRng(0, 0) draws exactly 0.0
    cdf = o.cdf_from_probs(o.marginal_probs(np.array([0, 2], dtype=complex), 1, [0]))
    assert o.partition_point(cdf, 0.0) == 1
    cdf_empty = o.cdf_from_probs(o.marginal_probs(np.array([0, 2], dtype=complex), 1, []))
    assert len(cdf_empty) == 1 and o.partition_point(cdf_empty, 0.0) == 0
    counts = o.sample_counts(np.array([2, 2], dtype=complex), 1, 10_000, 123)
    assert sum(counts.values()) == 10_000
    assert abs(counts["0"] - 5000) < 250
    assert "" in o.sample_counts(np.array([1], dtype=complex), 0, 1, 123, [])


@pytest.mark.parametrize("n", [1, 12])
def test_measurement_normalizes_both_branches_and_high_targets(n):
    # src/engine.rs:733-754; StepRng(0) draws 0.0, StepRng(u64::MAX) draws (2^53-1)/2^53
    hi_draw = o.lib().orc_u64_to_f64((1 << 64) - 1)
    for target in (0, n - 1):
        for outcome in (0, 1):
            s = np.zeros(1 << n, dtype=np.complex128)
            s[0] = 2.0
            s[1 << target] = 2.0
            draw = 0.0 if outcome == 1 else hi_draw
            got = o.lib().orc_measure(o._ptr(s), n, target, draw, 1, None)
            assert got == outcome
            assert abs(np.sum(np.abs(s) ** 2) - 1.0) < 1e-14
            assert s[outcome << target] == 1.0
            again = o.lib().orc_measure(o._ptr(s), n, target, o.ChaCha8Stream(9).gen_f64(), 0, None)
            assert again == outcome


def _apply_elementary(state, n, gate, target, controls):
    """src/gates.rs:306-319 (MSB-first wire order)."""
    bit = 1 << (n - 1 - target)
    cmask = 0
    for q in controls:
        cmask |= 1 << (n - 1 - q)
    for low in range(len(state)):
        if low & bit == 0 and low & cmask == cmask:
            high = low | bit
            a, b = state[low], state[high]
            state[low] = gate[0][0] * a + gate[0][1] * b
            state[high] = gate[1][0] * a + gate[1][1] * b


def _rccx_decomposition(state, n, first, extra):
    # src/gates.rs:321-342
    target = first + 2
    fc, sc = list(extra) + [first], list(extra) + [first + 1]
    for gate, ctl in ((o.h(), extra), (o.t_gate(), extra), (o.X, sc), (o.tdg(), extra), (o.X, fc),
                      (o.t_gate(), extra), (o.X, sc), (o.tdg(), extra), (o.h(), extra)):
        _apply_elementary(state, n, gate, target, ctl)


def test_rccx_and_rc3x_match_elementary_decompositions():
    # src/gates.rs:344-377
    m = o.rccx()
    for col in range(8):
        s = [0j] * 8
        s[col] = 1 + 0j
        _rccx_decomposition(s, 3, 0, [])
        for row in range(8):
            assert abs(s[row] - m[row][col]) < 1e-12
    m = o.rc3x()
    for col in range(16):
        s = [0j] * 16
        s[col] = 1 + 0j
        _rccx_decomposition(s, 4, 1, [0])
        _apply_elementary(s, 4, o.s_gate(), 1, [0])
        for row in range(16):
            assert abs(s[row] - m[row][col]) < 1e-12


def _ops(insts):
    return o.compile_ops([o.parse_instruction(i) for i in insts])


def test_terminal_sampling_keeps_correlations_and_last_classical_write():
    # src/monolithic/statevector/shots.rs:268-287
    ops = _ops([inst("h", qubit=0), inst("cx", control=0, target=1), inst("measure", qubit=0, cbit=0),
                inst("measure", qubit=1, cbit=1), inst("measure", qubit=1, cbit=2)])
    out = o.run_shots(ops, 2, 3, 1024, 5, 1024, None, True)
    assert out["strategy"] == "terminal_sampling"
    assert sum(out["counts"].values()) == 1024
    assert set(out["counts"]) == {"000", "111"}


def test_memory_budget_selects_one_worker_and_sampling_fallback():
    # src/monolithic/statevector/shots.rs:289-301
    ops = _ops([inst("h", qubit=0), inst("measure", qubit=0, cbit=0)])
    out = o.run_shots(ops, 2, 1, 10, 5, 65, 8, True)
    assert out["strategy"] == "trajectories"
    assert out["parallel_shots"] == 1
    assert out["working_bytes"] == 65
    with pytest.raises(MemoryError):
        o.run_shots(ops, 2, 1, 10, 5, 64, None, True)


def test_overflowing_state_size_rejected_without_allocating():
    # src/monolithic/statevector/shots.rs:303-307
    for n in (64, 61):
        with pytest.raises(MemoryError):
            o.state_layout(n)


def _regs(*specs):
    return {name: {"name": name, "base": base, "size": size} for name, base, size in specs}


def _validate(instructions, qregs=None, cregs=None):
    c = {"qregs": qregs or _regs(("q", 0, 3)), "cregs": cregs or _regs(("c", 0, 3)),
         "instructions": [o.parse_instruction(i) for i in instructions]}
    o.validate_circuit(c)


@pytest.mark.parametrize("case", GOLDEN["validation_accept"])
def test_validation_accepts(case):
    # src/monolithic/statevector/validation.rs:56-149
    _validate(case["instructions"], case.get("qregs"), case.get("cregs"))


@pytest.mark.parametrize("case", GOLDEN["validation_reject"])
def test_validation_rejects(case):
    # src/monolithic/statevector/validation.rs:75-199
    with pytest.raises(ValueError):
        _validate(case["instructions"], case.get("qregs"), case.get("cregs"))


def test_chacha_block_matches_chacha20_of_cryptography():
    """The ChaCha block function (word layout, rotations, feed-forward) against a
    second implementation; ChaCha8 is the same function with 4 double rounds."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms

    rng = np.random.default_rng(3)
    for _ in range(8):
        key = bytes(rng.integers(0, 256, size=32, dtype=np.uint8))
        words12 = [int(x) for x in rng.integers(0, 2**32, size=4, dtype=np.uint64)]
        ks = Cipher(algorithms.ChaCha20(key, struct.pack("<4I", *words12)), mode=None).encryptor().update(bytes(64))
        inw = np.array([0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(struct.unpack("<8I", key)) + words12,
                       dtype=np.uint32)
        out = np.zeros(16, dtype=np.uint32)
        o.lib().orc_chacha_block_words(inw.ctypes.data_as(ctypes.c_void_p), 10, out.ctypes.data_as(ctypes.c_void_p))
        assert out.tobytes() == ks


def test_rng_draws_are_uniform_and_stream_consistent():
    draws = o.first_draws(77, 20000)
    assert draws.min() >= 0.0 and draws.max() < 1.0
    assert abs(draws.mean() - 0.5) < 0.01
    stream = o.stream_draws(77, 20)
    seq = o.ChaCha8Stream(77)
    assert [seq.gen_f64() for _ in range(20)] == stream.tolist()
    assert stream[0] == draws[0]


# ---- tests/test_statevector.py:53-347 against the oracle ----
def sim(**kw):
    return o.OracleSimulator(**kw)


def test_little_endian_statevector_and_ordered_marginals():
    r = sim(seed=1729).simulate(Circuit(4, [inst("x", qubit=0), inst("x", qubit=2)]))
    expected = np.zeros(16, dtype=complex)
    expected[5] = 1
    np.testing.assert_allclose(r.statevector, expected, atol=1e-14)
    assert r.probabilities() == {5: 1.0}
    assert r.probabilities([0, 1]) == {2: 1.0}
    assert r.probabilities([1, 0]) == {1: 1.0}
    assert r.probabilities([]) == {0: 1.0}
    assert r.counts(shots=17, qubits=[0, 1], seed=2) == {"10": 17}
    assert r.counts(shots=17, qubits=[], seed=2) == {"": 17}


def test_full_and_marginal_probabilities_match_amplitudes():
    r = sim(seed=1729).simulate(Circuit(5, [inst("ry", qubit=0, theta=0.7), inst("h", qubit=4),
                                           inst("cx", control=4, target=2), inst("rx", qubit=1, theta=-0.3),
                                           inst("rxx", a=1, b=3, theta=0.8)]))
    probs = np.abs(r.statevector) ** 2
    actual = r.probabilities()
    np.testing.assert_allclose([actual.get(i, 0) for i in range(32)], probs, atol=1e-14)
    for qubits in ([3, 0, 4], [0], [4, 3, 2, 1, 0], []):
        expected = np.zeros(1 << len(qubits))
        for index, p in enumerate(probs):
            key = 0
            for q in qubits:
                key = (key << 1) | ((index >> q) & 1)
            expected[key] += p
        got = r.probabilities(qubits)
        np.testing.assert_allclose([got.get(i, 0) for i in range(len(expected))], expected, atol=1e-14)


def test_tiny_rotations_are_not_discarded_by_fusion():
    theta = 1e-11
    r = sim(seed=1729).simulate(Circuit(1, [inst("rx", qubit=0, theta=theta)]))
    np.testing.assert_allclose(r.statevector, [math.cos(theta / 2), -1j * math.sin(theta / 2)], rtol=1e-13,
                               atol=1e-15)


@pytest.mark.parametrize("sample_terminal", [True, False])
def test_terminal_sampling_preserves_joint_correlations_and_mapping(sample_terminal):
    c = Circuit(3, [inst("h", qubit=0), inst("cx", control=0, target=2), inst("measure", qubit=2, cbit=1),
                    inst("barrier"), inst("measure", qubit=0, cbit=3)], cbits=5)
    s = sim(seed=10, sample_terminal=sample_terminal)
    counts = s.simulate_shots(c, 4096)
    assert_distribution(counts, {"00000": 0.5, "01010": 0.5}, 4096)
    assert counts == s.simulate_shots(c, 4096)


@pytest.mark.parametrize("sample_terminal", [True, False])
def test_mid_circuit_measurement_and_feedback(sample_terminal):
    c = Circuit(2, [inst("h", qubit=0), inst("measure", qubit=0, cbit=0), conditional(inst("x", qubit=1), 1),
                    inst("x", qubit=0), inst("measure", qubit=0, cbit=1), inst("measure", qubit=1, cbit=2)], cbits=3)
    counts = sim(seed=15, sample_terminal=sample_terminal).simulate_shots(c, 4096)
    assert_distribution(counts, {"010": 0.5, "101": 0.5}, 4096)


def test_reset_and_nested_classical_conditionals():
    c = Circuit(2, [inst("x", qubit=0), inst("measure", qubit=0, cbit=2), inst("reset", qubit=0),
                    inst("measure", qubit=0, cbit=0),
                    conditional(conditional(inst("x", qubit=1), 0), 2, base=1, size=2),
                    inst("measure", qubit=1, cbit=1)], cbits=3)
    r = sim(seed=1729).simulate(c)
    assert r.classical_bits == {0: 0, 1: 1, 2: 1}
    np.testing.assert_allclose(r.statevector, [0, 0, 1, 0], atol=1e-14)
    assert sim(seed=22).simulate_shots(c, 64) == {"110": 64}

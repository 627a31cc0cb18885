"""GPU parity of the complex128 path against the CPU oracle, through the C ABI.

Amplitudes: <= 1e-12 max abs error (the reference's own tolerance,
src/engine.rs:526-531).  Measurements and sampling use the same ChaCha8
streams as the oracle, so seeded outcomes and counts are compared exactly.
"""

import math

import numpy as np
import pytest

from helpers import (GATES, Circuit, assert_distribution, brickwork, conditional, inst, qft, random_circuit)
from oracle import oracle as o

import dqsim

pytestmark = pytest.mark.gpu
TOL = 1e-12


def both(circuit, seed=1729, **kw):
    got = dqsim.StatevectorSimulator(seed=seed, max_memory_mb=1 << 16, **kw).simulate(circuit)
    want = o.OracleSimulator(seed=seed, max_memory_mb=1 << 16).simulate(circuit)
    return got, want


def max_err(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def entangled_prefix(n, rng):
    ins = []
    for q in range(n):
        ins.append(inst("u", qubit=q, theta=float(rng.uniform(0, 3)), phi=float(rng.uniform(-2, 2)),
                        lam=float(rng.uniform(-2, 2))))
    for q in range(n - 1):
        ins.append(inst("cx", control=q, target=q + 1))
    return ins


@pytest.mark.parametrize("n", [4, 5, 12, 13])
def test_every_gate_on_entangled_states_and_permuted_qubits(n):
    rng = np.random.default_rng(n)
    for kind, names, params in GATES:
        if len(names) > n:
            continue
        for placement in (list(range(len(names))), list(range(n - 1, n - 1 - len(names), -1)),
                          rng.choice(n, size=len(names), replace=False).tolist()):
            g = inst(kind, **dict(zip(names, placement)))
            for p in params:
                g[p] = float(rng.uniform(-math.pi, math.pi))
            c = Circuit(n, entangled_prefix(n, rng) + [g])
            got, want = both(c)
            assert max_err(got.statevector, want.statevector) <= TOL, (kind, placement)


@pytest.mark.parametrize("n,seed", [(5, 0), (5, 1), (9, 2), (13, 3), (16, 4)])
def test_random_circuits_of_all_gates(n, seed):
    c = Circuit(n, random_circuit(seed, n, 150))
    got, want = both(c)
    assert max_err(got.statevector, want.statevector) <= TOL


def test_brickwork_20q_depth20_amplitudes_and_chi_square():
    """The plain-form CPU-runnable workload: 20-qubit depth-20 U3+CX brickwork from seed 0, with shot
    histograms checked by a chi-square test against |amplitude|^2."""
    c = brickwork(20, 20, seed=0, measure=False)
    got, want = both(c)
    sv = got.statevector
    assert max_err(sv, want.statevector) <= TOL
    assert abs(np.sum(np.abs(sv) ** 2) - 1.0) < 1e-12
    # chi-square on the marginal of the low 6 qubits (64 pooled bins, >= 5 expected each at 20k shots)
    shots = 20000
    measured = brickwork(20, 20, seed=0, measure=True)
    counts = dqsim.StatevectorSimulator(seed=11, max_memory_mb=1 << 12).simulate_shots(measured, shots)
    assert sum(counts.values()) == shots
    probs = np.abs(want.statevector) ** 2
    low = np.bincount(np.arange(1 << 20) & 63, weights=probs, minlength=64)
    obs = np.zeros(64)
    for key, cnt in counts.items():
        obs[int(key, 2) & 63] += cnt
    exp = low * shots
    chi2 = float(np.sum((obs - exp) ** 2 / exp))
    # 63 degrees of freedom: p < 1e-6 beyond ~125
    assert chi2 < 125, chi2


def test_terminal_sampling_counts_equal_oracle_streams():
    c = brickwork(10, 8, seed=3, measure=True)
    for seed in (5, 2**63 + 7):
        got = dqsim.StatevectorSimulator(seed=seed).simulate_shots(c, 3000)
        want = o.OracleSimulator(seed=seed).simulate_shots(c, 3000)
        assert got == want


def test_trajectory_counts_equal_oracle_streams():
    ins = brickwork(6, 3, seed=4, measure=False).data["instructions"]
    ins += [inst("measure", qubit=0, cbit=0), conditional(inst("x", qubit=3), 1),
            inst("reset", qubit=1), inst("h", qubit=1), inst("measure", qubit=1, cbit=1),
            conditional(inst("ry", qubit=2, theta=0.7), 1, base=1), inst("measure", qubit=2, cbit=2),
            inst("measure", qubit=3, cbit=3)]
    c = Circuit(6, ins, 4)
    for workers in (None, 1, 3):
        got = dqsim.StatevectorSimulator(seed=9, max_parallel_shots=workers).simulate_shots(c, 500)
        want = o.OracleSimulator(seed=9).simulate_shots(c, 500)
        assert got == want


def test_single_trajectory_with_measurements_matches_oracle():
    ins = random_circuit(8, 7, 80, generic=False)
    ins += [inst("measure", qubit=2, cbit=0), conditional(inst("h", qubit=5), 1), inst("reset", qubit=4),
            inst("measure", qubit=5, cbit=1)]
    ins += random_circuit(9, 7, 40, generic=False)
    c = Circuit(7, ins, 2)
    for seed in range(6):
        got, want = both(c, seed=seed)
        assert got.classical_bits == want.classical_bits
        assert max_err(got.statevector, want.statevector) <= 1e-11


def test_result_queries_match_oracle():
    c = Circuit(9, random_circuit(21, 9, 120))
    got, want = both(c)
    for qubits in (None, [3, 0, 8], [0], [8, 7, 6, 5, 4, 3, 2, 1, 0], [], [1, 2, 3, 4, 5, 6, 7, 8, 0]):
        a, b = got.probabilities(qubits), want.probabilities(qubits)
        keys = set(a) | set(b)
        assert max(abs(a.get(k, 0) - b.get(k, 0)) for k in keys) < 1e-14
    for qubits in (None, [4, 1], []):
        assert got.counts(shots=4000, qubits=qubits, seed=77) == want.counts(shots=4000, qubits=qubits, seed=77)
    other = want.statevector
    assert abs(got.fidelity(other) - 1.0) < 1e-12
    assert got.fidelity(np.zeros(4, dtype=complex)) == 0.0


# ---- tests/test_statevector.py:53-347 of the reference, against the product ----
def simulate(circuit, **options):
    return dqsim.StatevectorSimulator(seed=1729, **options).simulate(circuit)


def test_little_endian_statevector_and_ordered_marginals():
    r = simulate(Circuit(4, [inst("x", qubit=0), inst("x", qubit=2)]))
    expected = np.zeros(16, dtype=complex)
    expected[5] = 1
    np.testing.assert_allclose(r.statevector, expected, atol=1e-14)
    assert r.probabilities() == {5: 1.0}
    assert r.probabilities([0, 1]) == {2: 1.0}
    assert r.probabilities([1, 0]) == {1: 1.0}
    assert r.probabilities([]) == {0: 1.0}
    assert r.counts(shots=17, qubits=[0, 1], seed=2) == {"10": 17}
    assert r.counts(shots=17, qubits=[], seed=2) == {"": 17}


def test_tiny_rotations_are_not_discarded_by_fusion():
    theta = 1e-11
    r = simulate(Circuit(1, [inst("rx", qubit=0, theta=theta)]))
    np.testing.assert_allclose(r.statevector, [math.cos(theta / 2), -1j * math.sin(theta / 2)], rtol=1e-13,
                               atol=1e-15)


def test_relative_controlled_x_gates_flip_the_target():
    for kind, controls in (("rccx", 2), ("rc3x", 3)):
        gate = inst(kind, target=controls)
        gate.update({f"control{i + 1}": i for i in range(controls)})
        r = simulate(Circuit(controls + 1, [*(inst("x", qubit=i) for i in range(controls)), gate]))
        assert abs(r.probabilities().get((1 << (controls + 1)) - 1, 0) - 1.0) < 1e-12


@pytest.mark.parametrize("sample_terminal", [True, False])
def test_terminal_sampling_preserves_joint_correlations_and_mapping(sample_terminal):
    c = Circuit(3, [inst("h", qubit=0), inst("cx", control=0, target=2), inst("measure", qubit=2, cbit=1),
                    inst("barrier"), inst("measure", qubit=0, cbit=3)], cbits=5)
    s = dqsim.StatevectorSimulator(seed=10, sample_terminal=sample_terminal)
    counts = s.simulate_shots(c, shots=4096)
    assert_distribution(counts, {"00000": 0.5, "01010": 0.5}, 4096)
    assert counts == s.simulate_shots(c, shots=4096)


@pytest.mark.parametrize("sample_terminal", [True, False])
def test_repeated_measurements_and_overwritten_classical_bits(sample_terminal):
    c = Circuit(3, [inst("h", qubit=0), inst("x", qubit=1), inst("measure", qubit=0, cbit=0),
                    inst("measure", qubit=0, cbit=2), inst("measure", qubit=1, cbit=0),
                    inst("measure", qubit=0, cbit=1)], cbits=3)
    counts = dqsim.StatevectorSimulator(seed=21, sample_terminal=sample_terminal).simulate_shots(c, shots=4096)
    assert_distribution(counts, {"001": 0.5, "111": 0.5}, 4096)


@pytest.mark.parametrize("sample_terminal", [True, False])
def test_mid_circuit_measurement_and_feedback(sample_terminal):
    c = Circuit(2, [inst("h", qubit=0), inst("measure", qubit=0, cbit=0), conditional(inst("x", qubit=1), 1),
                    inst("x", qubit=0), inst("measure", qubit=0, cbit=1), inst("measure", qubit=1, cbit=2)], cbits=3)
    s = dqsim.StatevectorSimulator(seed=15, sample_terminal=sample_terminal)
    counts = s.simulate_shots(c, shots=4096)
    assert_distribution(counts, {"010": 0.5, "101": 0.5}, 4096)
    assert counts == s.simulate_shots(c, shots=4096)


def test_reset_and_nested_classical_conditionals():
    c = Circuit(2, [inst("x", qubit=0), inst("measure", qubit=0, cbit=2), inst("reset", qubit=0),
                    inst("measure", qubit=0, cbit=0),
                    conditional(conditional(inst("x", qubit=1), 0), 2, base=1, size=2),
                    inst("measure", qubit=1, cbit=1)], cbits=3)
    r = simulate(c)
    assert r.classical_bits == {0: 0, 1: 1, 2: 1}
    np.testing.assert_allclose(r.statevector, [0, 0, 1, 0], atol=1e-14)
    assert dqsim.StatevectorSimulator(seed=22).simulate_shots(c, shots=64) == {"110": 64}


def test_reset_of_entangled_qubit_retains_other_qubits_mixture():
    c = Circuit(2, [inst("h", qubit=0), inst("cx", control=0, target=1), inst("reset", qubit=0),
                    inst("measure", qubit=0, cbit=0), inst("measure", qubit=1, cbit=1)], cbits=2)
    counts = dqsim.StatevectorSimulator(seed=24).simulate_shots(c, shots=4096)
    assert_distribution(counts, {"00": 0.5, "10": 0.5}, 4096)


def test_zero_shots_and_unwritten_classical_bits():
    for sample_terminal in (True, False):
        s = dqsim.StatevectorSimulator(seed=30, sample_terminal=sample_terminal)
        for cbits, outcome in ((0, ""), (3, "000")):
            c = Circuit(1, [inst("h", qubit=0)], cbits=cbits)
            assert s.simulate_shots(c, shots=0) == {}
            assert s.simulate_shots(c, shots=13) == {outcome: 13}


def test_result_sampling_is_seeded():
    r = simulate(Circuit(2, [inst("h", qubit=0), inst("cx", control=0, target=1)]))
    counts = r.counts(shots=4096, seed=77)
    assert counts == r.counts(shots=4096, seed=77)
    assert_distribution(counts, {"00": 0.5, "11": 0.5}, 4096)
    assert r.counts(shots=0) == {}


def test_invalid_probability_queries_fail():
    r = simulate(Circuit(2))
    for qubits in ([2], [0, 0], [1, 0, 1]):
        for method in (r.probabilities, r.counts):
            with pytest.raises(ValueError):
                method(qubits=qubits)


def test_worker_limit_preserves_seeded_trajectory_results():
    c = Circuit(2, [inst("h", qubit=0), inst("measure", qubit=0, cbit=0), conditional(inst("x", qubit=1), 1),
                    inst("measure", qubit=1, cbit=1)], cbits=2)
    counts = [dqsim.StatevectorSimulator(seed=38, max_memory_mb=1, max_parallel_shots=w,
                                         sample_terminal=False).simulate_shots(c, shots=257) for w in (1, 2, 4)]
    assert counts[0] == counts[1] == counts[2]


def test_wrapper_forwards_statevector_options():
    c = Circuit(1, [inst("x", qubit=0), inst("measure", qubit=0, cbit=0)], cbits=1)
    options = {"seed": 11, "max_memory_mb": 1, "max_parallel_shots": 1, "sample_terminal": False}
    r = dqsim.simulate_monolithic(c, **options)
    np.testing.assert_allclose(r.statevector, [0, 1], atol=1e-14)
    assert dqsim.simulate_monolithic_shots(c, shots=19, **options) == {"1": 19}


def test_profiles_confirm_terminal_sampling_and_dynamic_worker_budget(tmp_path, monkeypatch):
    import json

    monkeypatch.chdir(tmp_path)
    terminal = Circuit(2, [inst("h", qubit=0), inst("h", qubit=1), inst("measure", qubit=0, cbit=0),
                           inst("measure", qubit=1, cbit=1)], cbits=2)
    dynamic = Circuit(15, [inst("h", qubit=0), inst("measure", qubit=0, cbit=0),
                           conditional(inst("x", qubit=14), 1), inst("measure", qubit=14, cbit=1)], cbits=2)
    s = dqsim.StatevectorSimulator(seed=12, max_memory_mb=1)
    counts = s.simulate_shots(terminal, shots=4096, profile=True)
    assert_distribution(counts, {"00": .25, "01": .25, "10": .25, "11": .25}, 4096)
    data = json.loads(next((tmp_path / "dqsim_profiles").glob("*.json")).read_text())
    assert data["execution_strategy"] == "terminal_sampling"
    assert data["shot_times"] == []
    assert data["working_bytes"] <= 1024 ** 2
    s.simulate_shots(dynamic, shots=16, profile=True)
    data = json.loads(sorted((tmp_path / "dqsim_profiles").glob("*.json"))[-1].read_text())
    assert data["execution_strategy"] == "trajectories"
    assert data["parallel_shots"] == 1
    assert len(data["shot_times"]) == 16
    assert data["working_bytes"] <= 1024 ** 2


def test_simulation_profile_counts_executed_operations():
    c = Circuit(3, [inst("h", qubit=0), inst("cx", control=0, target=1), inst("measure", qubit=0, cbit=0),
                    conditional(inst("x", qubit=2), 1), inst("rzz", a=0, b=2, theta=0.4)], cbits=1)
    r = dqsim.StatevectorSimulator(seed=3, profile=True).simulate(c)
    p = r.profile
    executed = r.classical_bits[0]
    assert p.apply_one_qubit_calls == 1 + executed
    assert p.apply_n_qubit_calls == 2
    assert p.measure_qubit_calls == 1
    assert p.total_time > 0
    assert dqsim.StatevectorSimulator(seed=3).simulate(c).profile is None


def test_qft_and_large_state_norms():
    c = qft(14, seed=2)
    got, want = both(c)
    assert max_err(got.statevector, want.statevector) <= TOL
    big = brickwork(24, 3, seed=5, measure=False)
    got, want = both(big)
    assert max_err(got.statevector, want.statevector) <= TOL

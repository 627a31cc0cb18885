"""Batched uneven circuits: one persistent launch, tensor-core fused passes on side streams, and the CUDA
graph replay of both."""

import numpy as np
import pytest

from helpers import hea
from oracle import oracle as o

import dqsim
from dqsim import _core, workloads

pytestmark = pytest.mark.gpu
U64 = (1 << 64) - 1


def circuits(count, seed, qmin=5, qmax=15):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(qmin, qmax + 1))
        out.append(workloads.hea(n, int(rng.integers(2, 7)), seed=int(rng.integers(1 << 30)), measure=True))
    return out


def zz_of(sv):
    p = np.abs(sv) ** 2
    i = np.arange(len(p))
    return float(np.sum(np.where(((i ^ (i >> 1)) & 1) == 1, -p, p)))


@pytest.mark.parametrize("precision", ["complex128", "complex64"])
def test_batch_states_expectations_and_counts_match_oracle(precision):
    cs = circuits(20, 1)
    sim = dqsim.StatevectorSimulator(seed=99, precision=precision, max_memory_mb=1 << 14)
    b = _core.BatchedCircuits(sim, cs, shots=1024)
    b.run(use_graph=False)
    zz = b.expect_zz()
    for i, c in enumerate(cs):
        n = c.num_qubits
        unitary = workloads.TransportCircuit(n, [x for x in c.data["instructions"] if x["kind"] != "measure"])
        want = o.OracleSimulator(seed=1).simulate(unitary).statevector
        got = b.statevector(i, n)
        if precision == "complex128":
            assert np.max(np.abs(got - want)) <= 1e-12
            assert abs(zz[i] - zz_of(want)) <= 1e-12
            seed = (99 + i * _core.BATCH_SEED_STRIDE) & U64
            assert b.counts(i) == o.OracleSimulator(seed=seed).simulate_shots(c, 1024)
        else:
            assert abs(np.vdot(got, want)) ** 2 >= 1 - 1e-6
            assert abs(zz[i] - zz_of(want)) <= 1e-5
            assert sum(b.counts(i).values()) == 1024


def test_graph_replay_is_deterministic_and_matches_direct_run():
    cs = circuits(12, 2, 8, 17)
    sim = dqsim.StatevectorSimulator(seed=5, precision="complex64")
    b = _core.BatchedCircuits(sim, cs, shots=512)
    b.run(use_graph=False)
    direct = [b.counts(i) for i in range(len(cs))]
    zz0 = b.expect_zz()
    for _ in range(3):
        b.run(use_graph=True)
    assert [b.counts(i) for i in range(len(cs))] == direct
    np.testing.assert_array_equal(b.expect_zz(), zz0)
    assert b.passes >= len(cs)


def test_autotuned_batch_matches_default_plan():
    cs = circuits(6, 3, 12, 16)
    sim = dqsim.StatevectorSimulator(seed=6, precision="complex128")
    a = _core.BatchedCircuits(sim, cs, shots=256, autotune=True)
    d = _core.BatchedCircuits(sim, cs, shots=256)
    a.run()
    d.run()
    for i, c in enumerate(cs):
        assert np.max(np.abs(a.statevector(i, c.num_qubits) - d.statevector(i, c.num_qubits))) <= 1e-12


def test_batch_rejects_mid_circuit_measurement():
    from helpers import Circuit, inst

    c = Circuit(3, [inst("h", qubit=0), inst("measure", qubit=0, cbit=0), inst("x", qubit=1)], cbits=1)
    sim = dqsim.StatevectorSimulator(seed=1)
    with pytest.raises(ValueError):
        _core.BatchedCircuits(sim, [c], shots=16)


def test_tensor_core_batch_matches_oracle_and_replays_identically():
    """Complex64 circuits of 12 or more qubits as tensor-core fused passes on side streams (the smaller ones in
    the persistent kernel), captured in one graph: states, <Z0 Z1> and counts against the oracle."""
    cs = circuits(14, 4, 8, 18)
    sim = dqsim.StatevectorSimulator(seed=21, precision="complex64", max_memory_mb=1 << 14)
    b = _core.BatchedCircuits(sim, cs, shots=512, tensor_cores=True)
    w = b.work()
    assert w["fused_circuits"] == sum(1 for c in cs if c.num_qubits >= 12) > 0
    assert w["tensor_flops"] > 0 and w["bytes"] > 0
    b.run(use_graph=False)
    zz = b.expect_zz()
    direct = [b.counts(i) for i in range(len(cs))]
    for i, c in enumerate(cs):
        n = c.num_qubits
        unitary = workloads.TransportCircuit(n, [x for x in c.data["instructions"] if x["kind"] != "measure"])
        want = o.OracleSimulator(seed=1).simulate(unitary).statevector
        got = b.statevector(i, n)
        assert abs(np.vdot(got, want)) ** 2 >= 1 - 1e-6
        assert abs(zz[i] - zz_of(want)) <= 1e-5
        assert sum(direct[i].values()) == 512
    for _ in range(2):
        b.run(use_graph=True)
    assert [b.counts(i) for i in range(len(cs))] == direct
    np.testing.assert_array_equal(b.expect_zz(), zz)

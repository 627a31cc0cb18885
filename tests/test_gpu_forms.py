"""GPU parity of every execution form against the CPU oracle.

* per-gate complex128: one kernel per operation (the plain form);
* tiled complex128: shared-memory passes with fused <=3-qubit matrices, FP64;
* complex64: single-precision state, FP64 reductions; checked by state
  fidelity (>= 1 - 1e-6) and max amplitude error against the FP64 oracle.
"""

import numpy as np
import pytest

from helpers import Circuit, brickwork, conditional, hea, inst, qft, random_circuit
from oracle import oracle as o

import dqsim

pytestmark = pytest.mark.gpu


def run(circuit, **kw):
    return dqsim.StatevectorSimulator(seed=5, max_memory_mb=1 << 16, **kw).simulate(circuit).statevector


def oracle_sv(circuit):
    return o.OracleSimulator(seed=5, max_memory_mb=1 << 16).simulate(circuit).statevector


def fidelity(a, b):
    return abs(np.vdot(a, b)) ** 2


@pytest.mark.parametrize("execution", ["per_gate", "tiled"])
@pytest.mark.parametrize("n,seed", [(3, 0), (6, 1), (9, 2), (14, 3), (17, 4)])
def test_c128_forms_match_oracle(execution, n, seed):
    c = Circuit(n, random_circuit(seed, n, 200))
    want = oracle_sv(c)
    got = run(c, execution=execution)
    assert np.max(np.abs(got - want)) <= 1e-12


@pytest.mark.parametrize("m", [5, 7, 10, 12])
@pytest.mark.parametrize("fuse", [1, 2, 3])
def test_tile_shapes_and_fusion_widths(m, fuse):
    c = brickwork(16, 12, seed=m * 10 + fuse, measure=False)
    want = oracle_sv(c)
    got = run(c, execution="tiled", tile_qubits=m, fusion_width=fuse)
    assert np.max(np.abs(got - want)) <= 1e-12


def test_tiled_benchmark_families():
    for c in (qft(18, seed=1), hea(19, 8, seed=2), brickwork(20, 20, seed=0, measure=False)):
        want = oracle_sv(c)
        assert np.max(np.abs(run(c) - want)) <= 1e-12


def test_tiled_trajectories_with_mid_circuit_measurement():
    ins = brickwork(15, 4, seed=9, measure=False).data["instructions"]
    ins += [inst("measure", qubit=3, cbit=0), conditional(inst("h", qubit=14), 1),
            inst("reset", qubit=7)]
    ins += brickwork(15, 3, seed=10, measure=False).data["instructions"]
    ins += [inst("measure", qubit=q, cbit=q) for q in range(15)]
    c = Circuit(15, ins, 15)
    got = dqsim.StatevectorSimulator(seed=3, max_memory_mb=1 << 14).simulate_shots(c, 200)
    want = o.OracleSimulator(seed=3, max_memory_mb=1 << 14).simulate_shots(c, 200)
    assert got == want


@pytest.mark.parametrize("execution", ["per_gate", "tiled"])
def test_c64_fidelity_and_amplitude_error(execution):
    c = brickwork(20, 20, seed=0, measure=False)
    want = oracle_sv(c)
    got = run(c, precision="complex64", execution=execution)
    f = fidelity(got, want)
    err = float(np.max(np.abs(got - want)))
    assert f >= 1 - 1e-6, f
    assert err <= 1e-5, err


def test_c64_sampling_and_queries():
    c = brickwork(12, 10, seed=4, measure=True)
    got = dqsim.StatevectorSimulator(seed=8, precision="complex64").simulate_shots(c, 5000)
    assert sum(got.values()) == 5000
    r = dqsim.StatevectorSimulator(seed=8, precision="complex64").simulate(qft(10, seed=2))
    probs = r.probabilities()
    assert abs(sum(probs.values()) - 1.0) < 1e-5
    ref = oracle_sv(qft(10, seed=2))
    assert r.fidelity(ref) >= 1 - 1e-6


def phase_block_words(p):
    """16-byte words of a pass's phase block: 6 per phase, 2 per operation and one per matrix entry."""
    words = 6 * len(p["phases"])
    for ph in p["phases"]:
        for op in ph["ops"]:
            c, k = op["code"], op["k"]
            entries = (4 if c < 4 else 0 if c < 8 else 16 if c < 14 else 64 if c < 18 else 0 if c < 24
                       else 1 if c == 24 else 1 << k)
            words += 2 + entries
    return words


def test_phase_blocks_as_launch_arguments_and_in_device_memory():
    """complex128 tile passes take their phase block as a launch argument when it
    fits 2,040 words and read it from device memory otherwise: both reproduce the
    oracle."""
    from dqsim import _core

    small = brickwork(16, 12, seed=2, measure=False)
    large = brickwork(12, 40, seed=1, measure=False)  # one pass holds every operation
    sizes_small = [phase_block_words(p) for p in _core.tile_plan_dump(small.model_dump_json(), 12, 2)["passes"]]
    sizes_large = [phase_block_words(p) for p in _core.tile_plan_dump(large.model_dump_json(), 12, 2)["passes"]]
    assert max(sizes_small) <= 2040 < min(sizes_large)
    for c in (small, large):
        assert np.max(np.abs(run(c, execution="tiled", tile_qubits=12, fusion_width=2) - oracle_sv(c))) <= 1e-12

"""The complex64 fused form on tcgen05 tensor cores (fusion_width=5) against the
FP64 oracle: state fidelity >= 1 - 1e-6 and max amplitude error <= 1e-5."""

import numpy as np
import pytest

from helpers import Circuit, assert_distribution, brickwork, conditional, hea, inst, qft, random_circuit
from oracle import oracle as o

import dqsim
from dqsim import _core

pytestmark = pytest.mark.gpu


def fused(**kw):
    return dqsim.StatevectorSimulator(precision="complex64", fusion_width=5, max_memory_mb=1 << 16, **kw)


def check(circuit):
    got = fused(seed=3).simulate(circuit).statevector
    want = o.OracleSimulator(seed=3, max_memory_mb=1 << 16).simulate(circuit).statevector
    fid = abs(np.vdot(got, want)) ** 2
    err = float(np.max(np.abs(got - want)))
    assert fid >= 1 - 1e-6, fid
    assert err <= 1e-5, err
    return fid, err


@pytest.mark.parametrize("maker", [
    lambda: brickwork(12, 3, seed=1, measure=False),
    lambda: brickwork(14, 10, seed=2, measure=False),
    lambda: qft(16, seed=4),
    lambda: hea(18, 8, seed=5),
    lambda: brickwork(20, 20, seed=0, measure=False),
])
def test_fused_matches_oracle(maker):
    check(maker())


def test_fused_scattered_tile_uses_per_thread_copies():
    """A pass over qubits 0, 1 and every odd qubit up to 21 needs more than five
    TMA dimensions per box, so its tiles load by 16-byte copies instead."""
    from helpers import spread_brickwork

    c = spread_brickwork(24, [0, 1] + list(range(3, 22, 2)), 8, seed=3)
    assert not any(p["tma"]["ok"] for p in _core.fused_plan_dump(c.model_dump_json())["passes"])
    check(c)


@pytest.mark.parametrize("depth, withhold, blocks", [
    (10, 2, [7, 5, 1]),  # first pass cycles its gate images: an initial fetch withheld
    (10, 6, [7, 5, 1]),  # ... a fetch issued when step 1's buffer frees up
    (3, 2, [4, 1]),      # first pass holds all four gate images resident
])
def test_fused_bounded_wait_reports_and_recovers(depth, withhold, blocks):
    """A gate image that never arrives (its fetch withheld: a flag nothing sets)
    makes the kernel's bounded waits run out: the CTAs drain, free their tensor
    memory and set the error flag, the call raises RuntimeError, and the same
    simulator then runs normally.  Covers both gate-image modes: a ring (passes
    of more than five blocks) and resident images (five or fewer)."""
    c = brickwork(14, depth, seed=2, measure=False)
    assert [len(p["blocks"]) for p in _core.fused_plan_dump(c.model_dump_json())["passes"]] == blocks
    sim = fused(seed=3)
    try:
        _core.debug_fused_fault(withhold_step=withhold, wait_ms=20.0)
        with pytest.raises(RuntimeError, match="bounded wait"):
            sim.simulate(c)
    finally:
        _core.debug_fused_fault()
    got = sim.simulate(c).statevector
    want = o.OracleSimulator(seed=3, max_memory_mb=1 << 16).simulate(c).statevector
    assert abs(np.vdot(got, want)) ** 2 >= 1 - 1e-6


@pytest.mark.parametrize("maker", [lambda: brickwork(28, 40, seed=11, measure=False), lambda: qft(28, seed=12)])
def test_fused_at_scale_against_complex128_on_the_device(maker):
    """28 qubits (2 GiB complex64 against 4 GiB complex128 per-gate, compared on
    the device): depth-40 brickwork and QFT keep fidelity >= 1 - 1e-6 and max
    amplitude error <= 1e-5 through ~20 fused passes."""
    c = maker()
    got = _core.PreparedCircuit(fused(seed=1), c)
    got.run()
    ref = _core.PreparedCircuit(dqsim.StatevectorSimulator(seed=1, max_memory_mb=1 << 16, execution="per_gate"), c)
    ref.run()
    fid, err = got.compare(ref)
    assert abs(1 - fid) <= 1e-6 and err <= 1e-5, (fid, err)
    assert got.shape()["passes"] >= 10


@pytest.mark.parametrize("seed", range(3))
def test_fused_random_circuits(seed):
    check(Circuit(15, random_circuit(seed, 15, 200)))


def test_fused_trajectories_and_sampling():
    ins = brickwork(14, 4, seed=7, measure=False).data["instructions"]
    ins += [inst("measure", qubit=0, cbit=0), inst("reset", qubit=13), conditional(inst("x", qubit=13), 1),
            inst("measure", qubit=13, cbit=1)]
    ins += brickwork(14, 2, seed=8, measure=False).data["instructions"] + [inst("measure", qubit=5, cbit=2)]
    c = Circuit(14, ins, 3)
    counts = fused(seed=4).simulate_shots(c, 4000)
    want = o.OracleSimulator(seed=4).simulate_shots(c, 4000)
    assert sum(counts.values()) == 4000
    assert all(k[1] == k[2] for k in counts)  # the reset qubit copies the first outcome
    # same ChaCha8 streams; complex64 probabilities differ by ~1e-7, so almost every shot agrees
    tvd = sum(abs(counts.get(k, 0) - want.get(k, 0)) for k in set(counts) | set(want)) / 2 / 4000
    assert tvd < 0.01, (counts, want)
    plan = _core.PreparedCircuit(fused(seed=1), brickwork(22, 12, seed=3, measure=True), shots=5000)
    plan.run()
    assert plan.shape()["passes"] > 0
    ref = _core.PreparedCircuit(dqsim.StatevectorSimulator(seed=1, max_memory_mb=1 << 16),
                                brickwork(22, 12, seed=3, measure=True), shots=5000)
    ref.run()
    fid, err = plan.compare(ref)
    assert fid >= 1 - 1e-6 and err <= 1e-5


def test_repeated_calls_reuse_the_compiled_plan():
    """A simulator keeps the compiled operations and prefix executor of the circuit texts it ran: a repeated
    call skips parse, compile and planning and gives the counts a fresh simulator gives; other texts are
    planned on their own."""
    c = brickwork(14, 6, seed=3, measure=True)
    sim = dqsim.StatevectorSimulator(seed=5, precision="complex64")
    first = sim.simulate_shots(c, 4000)
    ph1 = _core.last_call_phases(sim)
    again = sim.simulate_shots(c, 4000)
    ph2 = _core.last_call_phases(sim)
    assert again == first
    assert ph1["parse"] > 0 and ph2["parse"] == 0 and ph2["compile"] == 0
    assert dqsim.StatevectorSimulator(seed=5, precision="complex64").simulate_shots(c, 4000) == first
    for s in range(6):  # more texts than the cache holds, then the first again
        other = brickwork(14, 6, seed=10 + s, measure=True)
        assert sim.simulate_shots(other, 500) == dqsim.StatevectorSimulator(
            seed=5, precision="complex64").simulate_shots(other, 500)
    assert sim.simulate_shots(c, 4000) == first
    assert _core.last_call_phases(sim)["parse"] > 0  # evicted, so planned again


@pytest.mark.parametrize("precision", ["complex128", "complex64"])
def test_sampling_workspace_follows_changing_sizes(precision):
    """A simulator keeps its terminal-sampling buffers (statevector, table, scratch, outcomes) between calls
    and reallocates them when a call needs other sizes: calls of changing qubit count, measured register and
    shot count on one simulator give the counts fresh simulators give, and only the first call of a size
    allocates."""
    def measured(n, qubits, seed):
        ins = brickwork(n, 5, seed=seed, measure=False).data["instructions"]
        return Circuit(n, ins + [inst("measure", qubit=q, cbit=c) for c, q in enumerate(qubits)], len(qubits))

    calls = [(measured(14, range(14), 1), 3000), (measured(16, range(16), 2), 3000),
             (measured(14, range(14), 1), 3000), (measured(14, [3, 9, 12], 4), 700),
             (measured(18, [0, 17, 5, 5], 6), 5000), (measured(14, range(14), 1), 3000)]
    sim = dqsim.StatevectorSimulator(seed=9, precision=precision)
    for i, (c, shots) in enumerate(calls):
        got = sim.simulate_shots(c, shots)
        assert got == dqsim.StatevectorSimulator(seed=9, precision=precision).simulate_shots(c, shots), i
        assert sum(got.values()) == shots
    again = sim.simulate_shots(calls[-1][0], calls[-1][1])
    assert _core.last_call_phases(sim)["table"] < 0.05  # same sizes as the call before: nothing allocated
    assert again == dqsim.StatevectorSimulator(seed=9, precision=precision).simulate_shots(*calls[-1])


def test_terminal_sampling_from_a_state_built_by_the_first_fused_pass():
    """Terminal sampling starts the unitary prefix from |0...0>; when its first step is a fused pass, that pass
    builds the input tiles itself (no state write, no load).  Counts follow the oracle's (same ChaCha8 streams;
    complex64 probabilities differ by ~1e-7, so almost every shot agrees), on one state and on a second call
    that reuses the workspace the first one left behind."""
    for seed, n in ((5, 14), (6, 16)):
        c = brickwork(n, 6, seed=seed, measure=True)
        sim = fused(seed=3)
        for _ in range(2):
            counts = sim.simulate_shots(c, 6000)
            want = o.OracleSimulator(seed=3).simulate_shots(c, 6000)
            tvd = sum(abs(counts.get(k, 0) - want.get(k, 0)) for k in set(counts) | set(want)) / 2 / 6000
            assert tvd < 0.01, tvd

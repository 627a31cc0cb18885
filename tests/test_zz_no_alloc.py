"""dq_measure_noalloc, the measurement entry point that allocates nothing.

Callers that cannot call cudaMalloc -- hosts whose device memory belongs to
their own budgeted allocator, and latency-bound loops that cannot pay for an
allocation's synchronisation -- hand it states already in device memory.
These tests check, through the C ABI, that two calls in a row give exactly
what the existing entry point (StatevectorSimulator.simulate with the same
seed) gives for the same measurements, that states written on a non-blocking
stream are measured correctly once that stream is synchronised, that a state
of zero norm fails the call without stopping the others, and that oversized
requests are refused.  The device buffers here are the test's own (torch);
the entry point itself allocates none.  This file is collected last, so a
failure here comes after every other test.
"""

import ctypes

import numpy as np
import pytest

from helpers import Circuit, inst, random_circuit

import dqsim
from dqsim import _core

pytestmark = pytest.mark.gpu
TOL = 1e-12


def measured(prefix, n, measures, seed, precision="complex128"):
    ins = list(prefix) + [inst("measure", qubit=q, cbit=c) for c, q in enumerate(measures)]
    sim = dqsim.StatevectorSimulator(seed=seed, precision=precision)
    return sim.simulate(Circuit(n, ins, cbits=max(1, len(measures))))


def device_copy(state):
    import torch

    return torch.from_numpy(np.ascontiguousarray(state)).to("cuda")


@pytest.mark.parametrize("seed", [7, 2**63 + 5])
def test_two_calls_match_simulate(seed):
    n, q1, q2 = 9, 3, 7
    prefix = random_circuit(11, n, 120, generic=False)
    before = dqsim.StatevectorSimulator(seed=seed).simulate(Circuit(n, prefix)).statevector
    t = device_copy(before)
    first = _core.measure_noalloc(t.data_ptr(), "complex128", 1, n, q1, seeds=[seed], draw_index=[0])
    r1 = measured(prefix, n, [q1], seed)
    assert first == [r1.classical_bits[0]]
    assert np.max(np.abs(t.cpu().numpy() - r1.statevector)) <= TOL
    second = _core.measure_noalloc(t.data_ptr(), "complex128", 1, n, q2, seeds=[seed], draw_index=[1])
    r2 = measured(prefix, n, [q1, q2], seed)
    assert second == [r2.classical_bits[1]]
    assert np.max(np.abs(t.cpu().numpy() - r2.statevector)) <= TOL


def test_batch_of_states_and_complex64():
    import torch

    n, q = 14, 12
    prefix = random_circuit(5, n, 80, generic=False)
    seeds = [3, 4, 5]
    before = dqsim.StatevectorSimulator(seed=1).simulate(Circuit(n, prefix)).statevector
    t = device_copy(np.concatenate([before] * 3))
    for call in range(2):
        out = _core.measure_noalloc(t.data_ptr(), "complex128", 3, n, q if call == 0 else 0, seeds=seeds,
                                    draw_index=[call] * 3)
        for i, s in enumerate(seeds):
            want = measured(prefix, n, [q] if call == 0 else [q, 0], s)
            assert out[i] == want.classical_bits[call]
            got = t[i << n:(i + 1) << n].cpu().numpy()
            assert np.max(np.abs(got - want.statevector)) <= TOL
    before64 = dqsim.StatevectorSimulator(seed=1, precision="complex64").simulate(Circuit(n, prefix)).statevector
    t64 = torch.from_numpy(before64.astype(np.complex64)).to("cuda")
    for call, qq in enumerate((q, 1)):
        out = _core.measure_noalloc(t64.data_ptr(), "complex64", 1, n, qq, seeds=[9], draw_index=[call])
        want = measured(prefix, n, [q, 1][:call + 1], 9, precision="complex64")
        assert out == [want.classical_bits[call]]
        assert np.max(np.abs(t64.cpu().numpy().astype(np.complex128) - want.statevector)) <= 1e-6


def test_requests_beyond_the_fixed_scratch_are_refused():
    import torch

    t = torch.zeros(16, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match="scratch"):
        _core.measure_noalloc(t.data_ptr(), "complex128", 64, 22, 0, seeds=[1] * 64, draw_index=[0] * 64)
    with pytest.raises(ValueError):
        _core.measure_noalloc(t.data_ptr(), "complex128", 1, 4, 9, seeds=[1], draw_index=[0])
    host = np.zeros(16, dtype=np.complex128)
    with pytest.raises(ValueError, match="device memory"):
        _core.measure_noalloc(host.ctypes.data, "complex128", 1, 4, 0, seeds=[1], draw_index=[0])


def test_states_written_on_a_non_blocking_stream():
    """The call runs on the legacy default stream, which does not wait for non-blocking streams: states
    written on one (torch's side streams are created non-blocking) are measured once it is synchronised."""
    import torch

    n, q1, q2 = 12, 5, 11
    prefix = random_circuit(21, n, 90, generic=False)
    before = dqsim.StatevectorSimulator(seed=3).simulate(Circuit(n, prefix)).statevector
    host = torch.from_numpy(np.ascontiguousarray(before)).pin_memory()
    t = torch.empty(1 << n, dtype=torch.complex128, device="cuda")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        t.copy_(host, non_blocking=True)
    side.synchronize()
    for call, qs in enumerate(([q1], [q1, q2])):
        out = _core.measure_noalloc(t.data_ptr(), "complex128", 1, n, qs[-1], seeds=[13], draw_index=[call])
        want = measured(prefix, n, qs, 13)
        assert out == [want.classical_bits[call]]
        assert np.max(np.abs(t.cpu().numpy() - want.statevector)) <= TOL


def test_zero_norm_state_fails_the_call_but_not_the_others():
    """A state of zero norm keeps outcome -1 and is left as it was; the call reports RuntimeError, and the
    other state of the call is measured and collapsed as the existing entry point does it."""
    n, q = 10, 4
    prefix = random_circuit(33, n, 60, generic=False)
    before = dqsim.StatevectorSimulator(seed=1).simulate(Circuit(n, prefix)).statevector
    t = device_copy(np.concatenate([before, np.zeros_like(before)]))
    seeds = np.array([17, 18], dtype=np.uint64)
    draws = np.zeros(2, dtype=np.uint64)
    out = np.full(2, 7, dtype=np.int32)
    status = _core._measure_noalloc(ctypes.c_void_p(t.data_ptr()), 0, 2, n, q, 0, seeds.ctypes.data_as(ctypes.c_void_p),
                                    draws.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    assert status == 4  # DQ_RUNTIME_ERROR
    assert "norm" in _core._last_error().decode()
    want = measured(prefix, n, [q], 17)
    assert out.tolist() == [want.classical_bits[0], -1]
    got = t.cpu().numpy()
    assert np.max(np.abs(got[:1 << n] - want.statevector)) <= TOL
    assert not np.any(got[1 << n:])

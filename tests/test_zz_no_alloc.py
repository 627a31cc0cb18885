"""dq_measure_noalloc, the measurement entry point that allocates nothing.

Callers that cannot call cudaMalloc -- code inside a CUDA stream capture,
hosts whose device memory belongs to their own budgeted allocator, and
latency-bound loops that cannot pay for an allocation's synchronisation --
hand it states already in device memory.  These tests check, through the C
ABI, that two calls in a row give exactly what the existing entry point
(StatevectorSimulator.simulate with the same seed) gives for the same
measurements, and that oversized requests are refused.  The device buffers
here are the test's own (torch); the entry point itself allocates none.
This file is collected last, so a failure here comes after every other test.
"""

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

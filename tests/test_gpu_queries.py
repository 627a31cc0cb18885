"""Device-side result queries beyond the reference's statevector result:
amplitude(s) and Pauli expectation values, against numpy on the oracle's state."""

import numpy as np
import pytest

from helpers import Circuit, brickwork, random_circuit
from oracle import oracle as o

import dqsim

pytestmark = pytest.mark.gpu

PAULI = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
         "Z": np.diag([1, -1])}


def numpy_expectation(state, pauli):
    """<psi|P|psi> with the string's first character on the highest qubit."""
    n = len(pauli)
    psi = state.reshape([2] * n)  # axis 0 = highest qubit (C order of the little-endian index)
    for axis, ch in enumerate(pauli):
        psi = np.moveaxis(np.tensordot(PAULI[ch], psi, axes=([1], [axis])), 0, axis)
    return complex(np.vdot(state, psi.reshape(-1)))


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-12), ("complex64", 1e-5)])
def test_amplitudes_and_expectations_match_numpy(precision, tol):
    rng = np.random.default_rng(7)
    for circuit in (brickwork(13, 6, seed=4, measure=False), Circuit(9, random_circuit(3, 9, 80))):
        n = circuit.data["qregs"]["q"]["size"]
        want = o.OracleSimulator(seed=2).simulate(circuit).statevector
        res = dqsim.StatevectorSimulator(seed=2, precision=precision).simulate(circuit)
        idx = rng.integers(0, 1 << n, size=50)
        np.testing.assert_allclose(res.amplitudes(idx), want[idx], atol=tol, rtol=0)
        for i in idx[:5]:
            bits = format(int(i), f"0{n}b")
            assert abs(res.amplitude(bits) - want[i]) <= tol
        for _ in range(12):
            pauli = "".join(rng.choice(list("IXYZ"), size=n))
            got = res.expectation_value(pauli)
            ref = numpy_expectation(want, pauli)
            assert abs(ref.imag) < 1e-12
            assert abs(got - ref.real) <= 10 * tol, (pauli, got, ref)


def test_query_validation_follows_the_reference_messages():
    res = dqsim.StatevectorSimulator(seed=1).simulate(brickwork(4, 2, seed=1, measure=False))
    for bad in ("010", "01010", "01a1"):
        with pytest.raises(ValueError, match="one binary digit per qubit"):
            res.amplitude(bad)
    with pytest.raises(ValueError, match="one Pauli per qubit"):
        res.expectation_value("XX")
    with pytest.raises(ValueError, match="only I, X, Y, Z"):
        res.expectation_value("XQZI")
    with pytest.raises(ValueError):
        res.amplitudes([16])
    assert res.expectation_value("IIII") == pytest.approx(1.0, abs=1e-12)

"""Circuit transport helpers and seeded circuit generators shared by the tests."""

import json
import math

import numpy as np

from dqsim import workloads


class Circuit:
    """Minimal transport object (tests/test_statevector.py:27-38 of the reference)."""

    def __init__(self, qubits, instructions=(), cbits=0):
        self.data = {
            "qregs": {"q": {"name": "q", "base": 0, "size": qubits}},
            "cregs": {"c": {"name": "c", "base": 0, "size": cbits}},
            "instructions": list(instructions),
        }

    def model_dump_json(self):
        return json.dumps(self.data)


def inst(kind, **fields):
    return {"kind": kind, **fields}


def conditional(op, value, base=0, size=1):
    return inst("conditional", condition={"creg_base": base, "creg_size": size, "creg_value": value}, op=op)


# (kind, operand names, parameter names) for every unitary instruction of src/types.rs.
GATES = [
    ("id", ("qubit",), ()), ("u0", ("qubit",), ()), ("x", ("qubit",), ()), ("y", ("qubit",), ()),
    ("z", ("qubit",), ()), ("h", ("qubit",), ()), ("s", ("qubit",), ()), ("sdg", ("qubit",), ()),
    ("t", ("qubit",), ()), ("tdg", ("qubit",), ()), ("sx", ("qubit",), ()), ("sxdg", ("qubit",), ()),
    ("u3", ("qubit",), ("theta", "phi", "lam")), ("u2", ("qubit",), ("phi", "lam")), ("u1", ("qubit",), ("lam",)),
    ("u", ("qubit",), ("theta", "phi", "lam")), ("p", ("qubit",), ("lam",)), ("rx", ("qubit",), ("theta",)),
    ("ry", ("qubit",), ("theta",)), ("rz", ("qubit",), ("phi",)),
    ("cx", ("control", "target"), ()), ("cz", ("control", "target"), ()), ("cy", ("control", "target"), ()),
    ("ch", ("control", "target"), ()), ("swap", ("a", "b"), ()), ("csx", ("control", "target"), ()),
    ("crx", ("control", "target"), ("theta",)), ("cry", ("control", "target"), ("theta",)),
    ("crz", ("control", "target"), ("lam",)), ("cu1", ("control", "target"), ("lam",)),
    ("cp", ("control", "target"), ("lam",)), ("cu3", ("control", "target"), ("theta", "phi", "lam")),
    ("cu", ("control", "target"), ("theta", "phi", "lam", "gamma")), ("rxx", ("a", "b"), ("theta",)),
    ("rzz", ("a", "b"), ("theta",)), ("ccx", ("control1", "control2", "target"), ()),
    ("cswap", ("control", "target1", "target2"), ()), ("rccx", ("control1", "control2", "target"), ()),
    ("rc3x", ("control1", "control2", "control3", "target"), ()),
    ("c3x", ("control1", "control2", "control3", "target"), ()),
    ("c3sqrtx", ("control1", "control2", "control3", "target"), ()),
    ("c4x", ("control1", "control2", "control3", "control4", "target"), ()),
]

GENERIC = [("remote_link_phi_plus", 2, 0), ("remote_link_psi_plus", 2, 0), ("remote_link_psi_minus", 2, 0),
           ("nonlocal_cz", 2, 0), ("remote_cz", 2, 0), ("remote_cx", 2, 0), ("remote_epr", 2, 0), ("epr", 2, 0),
           ("remote_rzz", 2, 1), ("remote_cu1", 2, 1), ("remote_barrier", 3, 0)]


def random_gate(rng, n):
    while True:
        kind, names, params = GATES[int(rng.integers(len(GATES)))]
        if len(names) <= n:
            break
    qubits = rng.choice(n, size=len(names), replace=False).tolist()
    out = inst(kind, **dict(zip(names, qubits)))
    for p in params:
        out[p] = float(rng.uniform(-math.pi, math.pi))
    return out


def random_generic(rng, n):
    name, arity, nparams = GENERIC[int(rng.integers(len(GENERIC)))]
    arity = min(arity, n)
    return inst("gate", name=name, qubits=rng.choice(n, size=arity, replace=False).tolist(),
                params=[float(rng.uniform(-3, 3)) for _ in range(nparams)])


def random_circuit(seed, n, depth, generic=True, barriers=True):
    rng = np.random.default_rng(seed)
    ins = []
    for _ in range(depth):
        r = rng.random()
        if generic and r < 0.05 and n >= 2:
            ins.append(random_generic(rng, n))
        elif barriers and r < 0.08:
            ins.append(inst("barrier"))
        else:
            ins.append(random_gate(rng, n))
    return ins


def brickwork(n, depth, seed=0, measure=True):
    return workloads.brickwork(n, depth, seed=seed, measure=measure)


def spread_brickwork(n, qubits, depth, seed=0):
    """Brickwork on a chosen set of qubits only (neighbours in the list are CX partners):
    a fused pass then has to hold exactly those qubits, however scattered they are."""
    rng = np.random.default_rng(seed)
    ins = []
    for layer in range(depth):
        for q in qubits:
            th, ph, la = (float(x) for x in rng.uniform(0.0, 2 * math.pi, size=3))
            ins.append(inst("u3", qubit=q, theta=th, phi=ph, lam=la))
        for i in range(layer % 2, len(qubits) - 1, 2):
            ins.append(inst("cx", control=qubits[i], target=qubits[i + 1]))
    return Circuit(n, ins)


def qft(n, seed=0):
    return workloads.qft(n, seed=seed)


def hea(n, depth, seed):
    return workloads.hea(n, depth, seed)


def assert_distribution(counts, expected, shots, delta=0.08):
    assert sum(counts.values()) == shots
    assert set(counts) == set(expected)
    for outcome, p in expected.items():
        assert abs(counts[outcome] / shots - p) <= delta, (outcome, counts[outcome] / shots, p)


def zz_expectation(statevector):
    """<Z0 Z1> of a statevector: sum of |a_i|^2 with sign -1 where qubits 0 and 1 differ."""
    p = np.abs(np.asarray(statevector)) ** 2
    idx = np.arange(p.shape[0])
    return float(np.dot(p, 1 - 2 * ((idx & 1) ^ ((idx >> 1) & 1))))

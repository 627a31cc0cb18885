"""Seeded synthetic circuits in the reference's transport schema.

The reference's headline workloads use public circuit suites it does not ship;
these generators stand in for them with the shapes and value distributions the
benchmark configurations state (numpy.random.default_rng(seed) throughout).
"""

import json
import math

import numpy as np


class TransportCircuit:
    """Anything with model_dump_json() is a circuit for StatevectorSimulator."""

    def __init__(self, qubits, instructions, cbits=0):
        self.num_qubits = qubits
        self.data = {
            "qregs": {"q": {"name": "q", "base": 0, "size": qubits}},
            "cregs": {"c": {"name": "c", "base": 0, "size": cbits}},
            "instructions": list(instructions),
        }
        self._text = None

    def model_dump_json(self):
        if self._text is None:
            self._text = json.dumps(self.data)
        return self._text


def brickwork(n, depth, seed=0, measure=True):
    """U3(theta, phi, lam) on every qubit with angles i.i.d. uniform [0, 2pi), then
    CX(2i, 2i+1) on even layers and CX(2i+1, 2i+2) on odd layers; measure all."""
    rng = np.random.default_rng(seed)
    ins = []
    for layer in range(depth):
        angles = rng.uniform(0.0, 2 * math.pi, size=(n, 3))
        for q in range(n):
            th, ph, la = (float(x) for x in angles[q])
            ins.append({"kind": "u3", "qubit": q, "theta": th, "phi": ph, "lam": la})
        for a in range(layer % 2, n - 1, 2):
            ins.append({"kind": "cx", "control": a, "target": a + 1})
    if measure:
        ins += [{"kind": "measure", "qubit": q, "cbit": q} for q in range(n)]
    return TransportCircuit(n, ins, n if measure else 0)


def qft(n, seed=0, measure=False):
    """Seeded computational-basis product state with H on a random half of the
    qubits, then H and CP(2pi/2^k) for all pairs and the swap network."""
    rng = np.random.default_rng(seed)
    ins = [{"kind": "x", "qubit": q} for q in range(n) if rng.random() < 0.5]
    for q in sorted(rng.choice(n, size=n // 2, replace=False).tolist()):
        ins.append({"kind": "h", "qubit": q})
    for j in range(n - 1, -1, -1):
        ins.append({"kind": "h", "qubit": j})
        for k in range(j - 1, -1, -1):
            ins.append({"kind": "cp", "control": k, "target": j, "lam": 2 * math.pi / 2 ** (j - k + 1)})
    for q in range(n // 2):
        ins.append({"kind": "swap", "a": q, "b": n - 1 - q})
    if measure:
        ins += [{"kind": "measure", "qubit": q, "cbit": q} for q in range(n)]
    return TransportCircuit(n, ins, n if measure else 0)


def hea(n, depth, seed, measure=False):
    """Hardware-efficient ansatz: RY, RZ on every qubit, then a CZ ladder (i, i+1)."""
    rng = np.random.default_rng(seed)
    ins = []
    for _ in range(depth):
        angles = rng.uniform(0.0, 2 * math.pi, size=(n, 2))
        for q in range(n):
            ins.append({"kind": "ry", "qubit": q, "theta": float(angles[q, 0])})
            ins.append({"kind": "rz", "qubit": q, "phi": float(angles[q, 1])})
        for q in range(n - 1):
            ins.append({"kind": "cz", "control": q, "target": q + 1})
    if measure:
        ins += [{"kind": "measure", "qubit": q, "cbit": q} for q in range(n)]
    return TransportCircuit(n, ins, n if measure else 0)


def hea_batch(count=512, seed=0, qmin=12, qmax=22, dmin=4, dmax=16):
    """Uneven HEA batch: qubits ~ U{qmin..qmax}, depth ~ U{dmin..dmax}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(qmin, qmax + 1))
        d = int(rng.integers(dmin, dmax + 1))
        out.append(hea(n, d, seed=int(rng.integers(1 << 31)), measure=True))
    return out


def benchmark_layers(n, depth):
    """The layered circuit of the reference's statevector benchmark
    (benchmarks/statevector_benchmark.py:30-37): per layer RY(0.23 + 0.017 (q + layer))
    and RZ(-0.41 + 0.019 layer) on every qubit, then CX(q, q + 1) down the register."""
    ins = []
    for layer in range(depth):
        for q in range(n):
            ins.append({"kind": "ry", "qubit": q, "theta": 0.23 + 0.017 * (q + layer)})
            ins.append({"kind": "rz", "qubit": q, "phi": -0.41 + 0.019 * layer})
        for q in range(n - 1):
            ins.append({"kind": "cx", "control": q, "target": q + 1})
    return ins


def benchmark_cases():
    """The four cases of benchmarks/statevector_benchmark.py:60-76, as circuits:
    terminal 12 q (256 shots), dynamic 10 q with a mid-circuit measure and a
    conditional X (128 shots), unitary 16 q, and a 14-qubit uniform state whose
    full probability table is queried."""
    def measure_all(n):
        return [{"kind": "measure", "qubit": q, "cbit": q} for q in range(n)]

    dynamic = benchmark_layers(10, 3) + [
        {"kind": "measure", "qubit": 0, "cbit": 0},
        {"kind": "conditional", "condition": {"creg_base": 0, "creg_size": 1, "creg_value": 1},
         "op": {"kind": "x", "qubit": 9}},
    ] + benchmark_layers(10, 3) + measure_all(10)
    return {
        "terminal_12q_256shots": (TransportCircuit(12, benchmark_layers(12, 8) + measure_all(12), 12), 256),
        "dynamic_10q_128shots": (TransportCircuit(10, dynamic, 10), 128),
        "unitary_16q": (TransportCircuit(16, benchmark_layers(16, 8)), None),
        "full_probabilities_14q": (TransportCircuit(14, [{"kind": "h", "qubit": q} for q in range(14)]), None),
    }

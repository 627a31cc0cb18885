"""Shared-memory tile planner, checked on the CPU.

The planner (dependency-respecting pass selection, in-pass fusion, lowering to
tile-local operations) is host code; this test replays its plan with a numpy
emulation of the tile kernel's per-operation semantics and compares the final
state with the oracle to 1e-12.  No GPU needed.
"""

import numpy as np
import pytest

from helpers import Circuit, brickwork, hea, inst, qft, random_circuit
from oracle import oracle as o

from dqsim import _core

ONE, X, DIAG_ENTRY, DIAG_FULL, SWAP, DENSE = range(6)


def expand(j, ins):
    j = np.asarray(j, dtype=np.int64)
    for p in ins:
        low = (1 << p) - 1
        j = (j & low) | ((j & ~low) << 1)
    return j


def deposit(v, positions):
    v = np.asarray(v, dtype=np.int64)
    out = np.zeros_like(v)
    for b, p in enumerate(positions):
        out |= ((v >> b) & 1) << p
    return out


def apply_op(tiles, op, m, pool):
    t = op["type"]
    if t in (ONE, X):
        j = np.arange(1 << (m - len(op["ins"])))
        i0 = expand(j, op["ins"]) | op["fixed"]
        i1 = i0 | op["tbit"]
        a, b = tiles[:, i0].copy(), tiles[:, i1].copy()
        if t == X:
            tiles[:, i0], tiles[:, i1] = b, a
        else:
            u = [complex(*pool[op["mat"] + k]) for k in range(4)]
            tiles[:, i0] = u[0] * a + u[1] * b
            tiles[:, i1] = u[2] * a + u[3] * b
    elif t == DIAG_ENTRY:
        i = expand(np.arange(1 << (m - len(op["ins"]))), op["ins"]) | op["fixed"]
        tiles[:, i] *= complex(*pool[op["mat"]])
    elif t == DIAG_FULL:
        e = np.arange(1 << m)
        jj = np.zeros_like(e)
        for q in op["q"]:
            jj = (jj << 1) | ((e >> q) & 1)
        d = np.array([complex(*pool[op["mat"] + x]) for x in range(1 << op["k"])])
        tiles *= d[jj][None, :]
    elif t == SWAP:
        i = expand(np.arange(1 << (m - len(op["ins"]))), op["ins"]) | op["fixed"]
        x, y = i | op["lowbit"], i | op["highbit"]
        a = tiles[:, x].copy()
        tiles[:, x] = tiles[:, y]
        tiles[:, y] = a
    elif t == DENSE:
        k = op["k"]
        D = 1 << k
        base = expand(np.arange(1 << (m - k)), op["ins"])
        cols = base[:, None] | np.asarray(op["offs"])[None, :]
        M = np.array([complex(*pool[op["mat"] + x]) for x in range(D * D)]).reshape(D, D)
        v = tiles[:, cols]
        tiles[:, cols] = v @ M.T
    else:
        raise AssertionError(t)


def emulate(plan):
    n = plan["n"]
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    for p in plan["passes"]:
        T = p["qubits"]
        m = len(T)
        other = [q for q in range(n) if q not in T]
        idx = deposit(np.arange(1 << (n - m)), other)[:, None] | deposit(np.arange(1 << m), T)[None, :]
        tiles = state[idx]
        for op in p["ops"]:
            assert all(x < m for x in op["ins"]) and all(x < m for x in op["q"])
            apply_op(tiles, op, m, plan["pool"])
        state[idx] = tiles
    return state


def oracle_state(circuit):
    return o.OracleSimulator(seed=1).simulate(circuit).statevector


def tileable_circuit(seed, n, depth):
    ins = [g for g in random_circuit(seed, n, depth) if g.get("kind") != "rc3x"]
    return Circuit(n, ins)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("m,fuse", [(3, 1), (4, 2), (5, 3), (6, 2)])
def test_tile_plan_reproduces_the_oracle(seed, m, fuse):
    n = 7 + seed % 3
    c = tileable_circuit(seed, n, 90)
    text = c.model_dump_json()
    plan = _core.tile_plan_dump(text, m, fuse)
    ops = o.circuit_ops(text)[2]
    assert sum(p["raw"] for p in plan["passes"]) == len(ops)
    assert all(len(p["qubits"]) == min(max(m, 5), n) for p in plan["passes"])
    np.testing.assert_allclose(emulate(plan), oracle_state(c), atol=1e-12, rtol=0)


@pytest.mark.parametrize("maker", [lambda: brickwork(12, 10, seed=1, measure=False), lambda: qft(10, seed=3),
                                   lambda: hea(11, 6, seed=4)])
def test_tile_plan_on_benchmark_families(maker):
    c = maker()
    text = c.model_dump_json()
    plan = _core.tile_plan_dump(text, 6, 2)
    np.testing.assert_allclose(emulate(plan), oracle_state(c), atol=1e-12, rtol=0)
    raw = sum(p["raw"] for p in plan["passes"])
    assert len(plan["passes"]) < raw  # many operations share each pass


def test_brickwork_30q_pass_count():
    """The planner's pass count for the 30q depth-40 workload (no state needed)."""
    from dqsim import workloads

    c = workloads.brickwork(30, 40, seed=0, measure=False)
    plan = _core.tile_plan_dump(c.model_dump_json(), 12, 2)
    raw = sum(p["raw"] for p in plan["passes"])
    assert raw == 1162 + 580
    assert len(plan["passes"]) < raw / 8, len(plan["passes"])

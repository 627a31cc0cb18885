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


# ---------------------------------------------------------------------------
# Register phases (csrc/phased.cu): each phase loads, per slot, the 16 amplitudes
# at base | rb[v] into registers, applies its operations there and stores them.
# ---------------------------------------------------------------------------
PH_ONE, PH_X, PH_D2, PH_D3, PH_SWAP, PH_DIAG_ENTRY, PH_DIAG_FULL = 0, 4, 8, 14, 18, 24, 25
PAIRS = [(1, 0), (2, 0), (2, 1), (3, 0), (3, 1), (3, 2)]
TRIPLES = [(2, 1, 0), (3, 1, 0), (3, 2, 0), (3, 2, 1)]


def swizzle(e, g=3):
    e = np.asarray(e, dtype=np.int64)
    f = np.zeros_like(e)
    x = e >> g
    while np.any(x):
        f ^= x
        x >>= g
    return e ^ (f & ((1 << g) - 1))


def phase_slots(ph):
    s = np.arange(1 << len(ph["sb"]))
    base = np.zeros_like(s)
    pbase = np.zeros_like(s)
    for i, (b, pb) in enumerate(zip(ph["sb"], ph["psb"])):
        base |= ((s >> i) & 1) * b
        pbase ^= ((s >> i) & 1) * pb
    return base, pbase


def apply_phase_op(a, full, op, pool):
    """a: (tiles, slots, E) register entries; full: (slots, E) tile indices."""
    code, E = op["code"], a.shape[2]

    def cond(v):
        return ((full[:, v] & op["mask"]) == op["value"])[None, :] if op["mask"] else True

    def mat(D):
        return np.array([complex(*pool[op["mat"] + k]) for k in range(D * D)]).reshape(D, D)

    if code < PH_D2:
        t = code % 4
        for v in range(E):
            if v & (1 << t):
                continue
            w = v | (1 << t)
            x, y = a[:, :, v].copy(), a[:, :, w].copy()
            if code < PH_X:
                u = mat(2).ravel()
                nx, ny = u[0] * x + u[1] * y, u[2] * x + u[3] * y
            else:
                nx, ny = y, x
            c = cond(v)
            a[:, :, v] = np.where(c, nx, x)
            a[:, :, w] = np.where(c, ny, y)
    elif code < PH_D3:
        H, L = PAIRS[code - PH_D2]
        M = mat(4)
        for v in range(E):
            if v & ((1 << H) | (1 << L)):
                continue
            idx = [v | (((c >> 1) & 1) << H) | ((c & 1) << L) for c in range(4)]
            a[:, :, idx] = a[:, :, idx] @ M.T
    elif code < PH_SWAP:
        A, B, C = TRIPLES[code - PH_D3]
        M = mat(8)
        for v in range(E):
            if v & ((1 << A) | (1 << B) | (1 << C)):
                continue
            idx = [v | (((c >> 2) & 1) << A) | (((c >> 1) & 1) << B) | ((c & 1) << C) for c in range(8)]
            a[:, :, idx] = a[:, :, idx] @ M.T
    elif code < PH_DIAG_ENTRY:
        H, L = PAIRS[code - PH_SWAP]
        for v in range(E):
            if v & ((1 << H) | (1 << L)):
                continue
            v01, v10 = v | (1 << L), v | (1 << H)
            c = cond(v01)
            x, y = a[:, :, v01].copy(), a[:, :, v10].copy()
            a[:, :, v01] = np.where(c, y, x)
            a[:, :, v10] = np.where(c, x, y)
    elif code == PH_DIAG_ENTRY:
        d = complex(*pool[op["mat"]])
        for v in range(E):
            a[:, :, v] = np.where(cond(v), a[:, :, v] * d, a[:, :, v])
    elif code == PH_DIAG_FULL:
        table = np.array([complex(*pool[op["mat"] + x]) for x in range(1 << op["k"])])
        for v in range(E):
            jj = np.zeros(full.shape[0], dtype=np.int64)
            for q in op["q"]:
                jj = (jj << 1) | ((full[:, v] >> q) & 1)
            a[:, :, v] *= table[jj][None, :]
    else:
        raise AssertionError(code)


def emulate_phased(plan):
    n = plan["n"]
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    for p in plan["passes"]:
        T = p["qubits"]
        m = len(T)
        assert p["phases"], "every pass of at least 6 tile qubits runs in phases"
        assert sum(len(ph["ops"]) for ph in p["phases"]) == len(p["ops"])
        other = [q for q in range(n) if q not in T]
        idx = deposit(np.arange(1 << (n - m)), other)[:, None] | deposit(np.arange(1 << m), T)[None, :]
        tiles = state[idx]
        for ph in p["phases"]:
            base, pbase = phase_slots(ph)
            full = base[:, None] | np.asarray(ph["rb"])[None, :]
            # every tile index once per phase, and the swizzled addresses too
            assert sorted(full.ravel().tolist()) == list(range(1 << m))
            assert np.array_equal(pbase[:, None] ^ np.asarray(ph["prb"])[None, :], swizzle(full))
            a = tiles[:, full]
            for op in ph["ops"]:
                apply_phase_op(a, full, op, plan["pool"])
            tiles[:, full] = a
        state[idx] = tiles
    return state


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("m,fuse", [(6, 1), (6, 3), (7, 2), (8, 3)])
def test_register_phases_reproduce_the_oracle(seed, m, fuse):
    n = 7 + seed % 3
    c = tileable_circuit(seed, n, 90)
    plan = _core.tile_plan_dump(c.model_dump_json(), m, fuse)
    np.testing.assert_allclose(emulate_phased(plan), oracle_state(c), atol=1e-12, rtol=0)


@pytest.mark.parametrize("maker", [lambda: brickwork(12, 10, seed=1, measure=False), lambda: qft(10, seed=3),
                                   lambda: hea(11, 6, seed=4)])
def test_register_phases_on_benchmark_families(maker):
    c = maker()
    plan = _core.tile_plan_dump(c.model_dump_json(), 8, 2)
    np.testing.assert_allclose(emulate_phased(plan), oracle_state(c), atol=1e-12, rtol=0)


def test_register_phases_30q_brickwork_layout():
    """The 30q depth-40 plan: two or more operations per phase on average with
    three register qubits (3.5 with four), and the 8 lanes of every
    quarter-warp (slot bits 0-2) hit 8 distinct 16-byte bank groups."""
    from dqsim import workloads

    c = workloads.brickwork(30, 40, seed=0, measure=False)
    plan = _core.tile_plan_dump(c.model_dump_json(), 12, 2)
    ops = sum(len(p["ops"]) for p in plan["passes"])
    phases = sum(len(p["phases"]) for p in plan["passes"])
    entries = len(plan["passes"][0]["phases"][0]["rb"])
    assert ops >= (2.0 if entries == 8 else 3.5) * phases, (ops, phases)
    for p in plan["passes"]:
        for ph in p["phases"]:
            base, pbase = phase_slots(ph)
            for v in range(len(ph["rb"])):
                addr = pbase ^ ph["prb"][v]
                quarter = addr.reshape(-1, 8) & 7
                assert all(len(set(q.tolist())) == 8 for q in quarter)

"""The tensor-core fused plan, replayed on the CPU.

The host side of the fused complex64 form -- 12-qubit passes, 5-qubit block
fusion, the per-block layout tables (which TMEM column / tile row every output
amplitude goes to next) and the TF32 hi/lo gate images in the canonical
K-major operand layout -- is replayed here with numpy, block by block, exactly
as the kernel consumes it, and compared with the FP64 oracle.  No GPU needed.
"""

import struct

import numpy as np
import pytest

from helpers import Circuit, brickwork, hea, qft, random_circuit
from oracle import oracle as o

from dqsim import _core


def canon(row, k):
    return (row // 8) * 512 + (k // 4) * 32 + (row % 8) * 4 + k % 4


ROWS = np.arange(64)[:, None]
KS = np.arange(64)[None, :]
CANON = canon(ROWS, KS)


def deposit(v, positions):
    v = np.asarray(v, dtype=np.int64)
    out = np.zeros_like(v)
    for b, p in enumerate(positions):
        out |= ((v >> b) & 1) << p
    return out


def block_matrix(upool, off):
    hi = upool[off:off + 4096][CANON]
    lo = upool[off + 4096:off + 8192][CANON]
    real = hi.astype(np.float64) + lo.astype(np.float64)
    return real[0::2, 0::2] + 1j * real[1::2, 0::2]


def operand_offset(packed):
    """Byte offset of packed (column << 5) | basis in the 128-byte swizzled tile operand."""
    col, basis = packed >> 5, packed & 31
    return ((basis >> 4) * 16384 + (col >> 3) * 1024 + (col & 7) * 128 + ((((basis >> 1) & 7) ^ (col & 7)) << 4)
            + (basis & 1) * 8)


PACKED = np.arange(4096)
SLOT_OF_PACKED = operand_offset(PACKED) // 8  # operand slot holding packed position p


def emulate(plan):
    n = plan["n"]
    upool = np.asarray(plan["upool"], dtype=np.float32)
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    local = np.arange(4096)
    for p in plan["passes"]:
        T = p["qubits"]
        other = [q for q in range(n) if q not in T]
        idx = deposit(np.arange(1 << (n - 12)), other)[:, None] | deposit(local, T)[None, :]
        tiles = state[idx]
        # shared memory as 4096 eight-byte slots; tables hold byte offsets combined by XOR
        off = np.asarray(p["in_lo"])[local & 63] ^ np.asarray(p["in_hi"])[local >> 6]
        slots = np.zeros_like(tiles)
        slots[:, off // 8] = tiles
        for blk in p["blocks"]:
            X = slots[:, SLOT_OF_PACKED].reshape(-1, 128, 32)
            U = block_matrix(upool, blk["u_off"])
            Y = X @ U.T
            off = np.asarray(blk["next_c"])[:, None] ^ np.asarray(blk["next_b"])[None, :]
            slots = np.zeros_like(tiles)
            slots[:, off // 8] = Y
        out = np.asarray(p["out_lo"])[local & 63] ^ np.asarray(p["out_hi"])[local >> 6]
        tiles = slots[:, out // 8]
        state[idx] = tiles
    return state


def check(circuit):
    text = circuit.model_dump_json()
    plan = _core.fused_plan_dump(text)
    got = emulate(plan)
    want = o.OracleSimulator(seed=1).simulate(circuit).statevector
    fid = abs(np.vdot(got, want)) ** 2
    assert fid >= 1 - 1e-6, fid
    assert np.max(np.abs(got - want)) <= 1e-5
    return plan


@pytest.mark.parametrize("maker", [lambda: brickwork(14, 8, seed=3, measure=False), lambda: qft(13, seed=1),
                                   lambda: hea(15, 5, seed=2), lambda: brickwork(12, 4, seed=9, measure=False)])
def test_fused_plan_reproduces_the_oracle(maker):
    plan = check(maker())
    assert all(len(p["qubits"]) == 12 for p in plan["passes"])


@pytest.mark.parametrize("seed", range(3))
def test_fused_plan_random_circuits(seed):
    ins = [g for g in random_circuit(seed, 13, 120) if g.get("kind") not in ("barrier",)]
    check(Circuit(13, ins))


def test_gate_images_are_tf32_hi_lo_pairs():
    plan = _core.fused_plan_dump(brickwork(13, 4, seed=1, measure=False).model_dump_json())
    up = np.asarray(plan["upool"], dtype=np.float32)
    bits = up.view(np.uint32)
    for blk in plan["passes"][0]["blocks"]:
        hi = bits[blk["u_off"]:blk["u_off"] + 4096]
        assert np.all((hi & 0x1FFF) == 0)  # 10 explicit mantissa bits
    assert plan["passes"][0]["blocks"][-1]["last"] == 1


def test_fused_block_counts_for_30q_brickwork():
    from dqsim import workloads

    plan = _core.fused_plan_dump(workloads.brickwork(30, 40, seed=0, measure=False).model_dump_json())
    blocks = sum(len(p["blocks"]) for p in plan["passes"])
    assert len(plan["passes"]) < 40
    assert blocks < 1742 / 4, blocks

"""The tensor-core fused plan, replayed on the CPU.

The host side of the fused complex64 form -- 12-qubit passes, 5-qubit block
fusion, the per-block layout tables (where in the next block's swizzled
operand every output amplitude goes) and the f16 hi/lo gate images in the
K-major 128-byte swizzled operand layout -- is replayed here with numpy, block
by block, exactly as the kernel consumes it, and compared with the FP64
oracle.  No GPU needed.
"""

import struct

import numpy as np
import pytest

from helpers import Circuit, brickwork, hea, qft, random_circuit
from oracle import oracle as o

from dqsim import _core


def sw128_half(row, k):
    """Half-word index of (row, k) in a K-major, 128-byte swizzled f16 operand (64 K per row)."""
    byte = (row // 8) * 1024 + (row % 8) * 128 + (((k * 2) >> 4) ^ (row % 8)) * 16 + ((k * 2) & 15)
    return byte // 2


ROWS = np.arange(64)[:, None]
KS = np.arange(64)[None, :]
SW128 = sw128_half(ROWS, KS)


def deposit(v, positions):
    v = np.asarray(v, dtype=np.int64)
    out = np.zeros_like(v)
    for b, p in enumerate(positions):
        out |= ((v >> b) & 1) << p
    return out


def block_matrix(upool, off):
    """The block's 32x32 complex matrix from its f16 hi/lo gate image."""
    hi = upool[off:off + 4096][SW128].astype(np.float64)
    lo = upool[off + 4096:off + 8192][SW128].astype(np.float64)
    real = hi + lo
    return real[0::2, 0::2] + 1j * real[1::2, 0::2]


def operand_offset(packed):
    """Byte offset of packed (column << 5) | basis in the f16, 128-byte swizzled tile operand."""
    col, basis = packed >> 5, packed & 31
    return (col >> 3) * 1024 + (col & 7) * 128 + (((basis >> 2) ^ (col & 7)) << 4) + (basis & 3) * 4


PACKED = np.arange(4096)
SLOT_OF_PACKED = operand_offset(PACKED) // 4  # 4-byte operand slot holding packed position p


def tile_bases(T, n, tiles):
    other = [q for q in range(n) if q not in T]
    return ((tiles >> (n - 12)) << n) | deposit(tiles & ((1 << (n - 12)) - 1), other)


def random_circuit_n(n, gates, seed):
    ins = [g for g in random_circuit(seed, n, gates) if g.get("kind") not in ("barrier", "measure", "reset")]
    return Circuit(n, ins)


def split_tile(p, tiles):
    """The kernel's split of loaded tiles into block 0's operand: thread gt takes the
    pairs (e, e + 1), e = P(gt) | split_q[k], P depositing bits 1..7 of 2 * gt at
    split_pos, and stores them at split_off(gt) ^ split_qoff[k] (and ^ in_lo[1])."""
    in_lo, in_hi = np.asarray(p["in_lo"]), np.asarray(p["in_hi"])
    pos, q, qoff = p["split_pos"], np.asarray(p["split_q"]), np.asarray(p["split_qoff"])
    gt = np.arange(128)
    P = np.zeros(128, dtype=np.int64)
    for b in range(1, 8):
        P |= (((2 * gt) >> b) & 1) << pos[b]
    split_off = in_lo[P & 63] ^ in_hi[P >> 6]
    slots = np.zeros_like(tiles)
    seen = np.zeros(4096, dtype=np.int64)
    for k in range(16):
        e = P | q[k]
        off = split_off ^ qoff[k]
        assert np.array_equal(off, in_lo[e & 63] ^ in_hi[e >> 6])  # the per-iteration offsets are the layout's
        slots[:, off // 4] = tiles[:, e]
        slots[:, (off ^ in_lo[1]) // 4] = tiles[:, e + 1]
        seen[e] += 1
        seen[e + 1] += 1
    assert np.all(seen == 1)  # every amplitude of the tile exactly once
    return slots


def emulate(plan):
    n = plan["n"]
    upool = np.asarray(plan["upool"], dtype=np.uint16).view(np.float16)
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    local = np.arange(4096)
    for p in plan["passes"]:
        T = p["qubits"]
        other = [q for q in range(n) if q not in T]
        idx = deposit(np.arange(1 << (n - 12)), other)[:, None] | deposit(local, T)[None, :]
        tiles = state[idx]
        # tables hold byte offsets combined by XOR: 4-byte operand entries, 8-byte stage entries
        slots = split_tile(p, tiles)
        for blk in p["blocks"]:
            X = slots[:, SLOT_OF_PACKED].reshape(-1, 128, 32)
            U = block_matrix(upool, blk["u_off"])
            Y = X @ U.T
            off = np.asarray(blk["next_c"])[:, None] ^ np.asarray(blk["next_b"])[None, :]
            slots = np.zeros_like(tiles)
            slots[:, off // (8 if blk["last"] else 4)] = Y
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


def test_gate_images_are_f16_hi_lo_pairs():
    plan = _core.fused_plan_dump(brickwork(13, 4, seed=1, measure=False).model_dump_json())
    up = np.asarray(plan["upool"], dtype=np.uint16).view(np.float16)
    for blk in plan["passes"][0]["blocks"]:
        hi = up[blk["u_off"]:blk["u_off"] + 4096]
        lo = up[blk["u_off"] + 4096:blk["u_off"] + 8192]
        # lo is at most half an f16 unit of hi: it carries the next 11 bits
        assert np.all(np.abs(lo.astype(np.float64)) <= np.abs(hi.astype(np.float64)) * 2.0 ** -11 + 2.0 ** -24)
    assert plan["passes"][0]["blocks"][-1]["last"] == 1


def tma_tile(tma, base):
    """Global element index of each local index of the tile whose local index 0 is at `base`, as the TMA boxes load it."""
    dims, lo, box = tma["dims"], tma["lo"], tma["box"]
    coord = [(base >> lo[i]) & ((1 << tma["bits"][i]) - 1) for i in range(dims - 1)] + [base >> lo[dims - 1]]
    per_copy = tma["copy_bytes"] // 8
    out = np.empty(per_copy * tma["copies"], dtype=np.int64)
    e = np.arange(per_copy)
    for c in range(tma["copies"]):
        addr = np.zeros(per_copy, dtype=np.int64)
        rem = e.copy()
        for i in range(dims):  # box elements in row-major order, dimension 0 fastest
            k = rem % box[i]
            rem //= box[i]
            ci = coord[i] + (tma["copy_step"][c] if i == dims - 1 else 0)
            addr += (ci + k) << lo[i]
        out[c * per_copy:(c + 1) * per_copy] = addr
    return out


@pytest.mark.parametrize("maker", [lambda: brickwork(30, 40, seed=0, measure=False), lambda: qft(26, seed=0),
                                   lambda: hea(22, 8, seed=0), lambda: brickwork(14, 8, seed=3, measure=False),
                                   lambda: random_circuit_n(20, 400, 5)])
def test_tma_boxes_load_each_tile_in_natural_order(maker):
    plan = _core.fused_plan_dump(maker().model_dump_json())
    n = plan["n"]
    local = np.arange(4096)
    for p in plan["passes"]:
        tma = p["tma"]
        if not tma["ok"]:
            continue
        assert tma["dims"] <= 5 and max(tma["box"]) <= 256 and tma["copies"] <= 16
        assert all(b * 8 % 16 == 0 for b in tma["box"][:1])  # inner box side: whole 16-byte units
        assert tma["copy_bytes"] * tma["copies"] == 32768
        T = p["qubits"]
        for t in (0, 1, (1 << (n - 12)) - 1, 12345 % (1 << (n - 12))):
            base = int(tile_bases(T, n, np.array([t]))[0])
            assert np.array_equal(tma_tile(tma, base), base | deposit(local, T))
    assert any(p["tma"]["ok"] for p in plan["passes"])


def test_scattered_tiles_fall_back_to_per_thread_copies():
    from helpers import spread_brickwork

    scattered = [0, 1] + list(range(3, 22, 2))
    plan = _core.fused_plan_dump(spread_brickwork(24, scattered, 6, seed=1).model_dump_json())
    assert plan["passes"] and all(p["qubits"] == scattered for p in plan["passes"])
    assert not any(p["tma"]["ok"] for p in plan["passes"])
    check(spread_brickwork(16, [0, 1, 3, 5, 6, 7, 9, 10, 11, 13, 14, 15], 6, seed=2))


def test_operand_offsets_are_a_bijection():
    offs = operand_offset(PACKED)
    assert len(set(offs.tolist())) == 4096 and offs.max() < 16384 and np.all(offs % 4 == 0)


def test_fused_block_counts_for_30q_brickwork():
    from dqsim import workloads

    plan = _core.fused_plan_dump(workloads.brickwork(30, 40, seed=0, measure=False).model_dump_json())
    blocks = sum(len(p["blocks"]) for p in plan["passes"])
    # passes from a beam search over pass sequences, blocks from a beam search
    # over the 5-qubit sets that absorb the most operations (first-fit fusion
    # gave 141 blocks); the plan's estimated cost is 3 per pass + 1 per block
    # (24 passes and 107 blocks here; 23 and 117 from one pass at a time by the
    # fewest-new-qubits rule)
    assert blocks <= 110, blocks
    assert 3 * len(plan["passes"]) + blocks <= 180


def _spread(qubits, spread_bit=20, pinned=2, inflight=9):
    """A pass's spread in quarters: 4 per tile qubit from spread_bit + 4 up, 3
    per tile qubit in [spread_bit, spread_bit + 4), less 12 per tile qubit that
    lengthens the contiguous runs the tiles in flight read together."""
    T = set(qubits)
    top = sum(1 for q in T if q >= spread_bit + 4)
    mid = sum(1 for q in T if spread_bit <= q < spread_bit + 4)
    run = outside = 0
    for q in range(64):
        if q in T:
            run += q >= pinned
        else:
            outside += 1
            if outside > inflight:
                break
    return 4 * top + 3 * mid - 12 * run


def _plan_cost(plan):
    """3 per pass + 1 per block + 4 (8) per pass whose spread exceeds 24 by at
    most (more than) 4 quarters."""
    cost = 0.0
    for p in plan["passes"]:
        s = _spread(p["qubits"])
        cost += 3 + len(p["blocks"]) + (8 if s > 28 else 4 if s > 24 else 0)
    return cost


@pytest.mark.parametrize("name, cost_max", [("bw30", 180), ("qft30", 142), ("qft32", 165), ("hea26", 110)])
def test_pass_search_and_spread_cap(name, cost_max):
    """The lookahead growth rule and the beam over pass sequences (QFT at 30
    qubits took 33 passes and 114 blocks, HEA at 26 qubits 21 and 82, with the
    fewest-new-qubits rule alone), under the spread cap or with the spread
    priced in, whichever plan costs less."""
    from dqsim import workloads

    c = {"bw30": lambda: workloads.brickwork(30, 40, seed=0, measure=False),
         "qft30": lambda: workloads.qft(30, seed=0),
         "qft32": lambda: workloads.qft(32, seed=0),
         "hea26": lambda: workloads.hea(26, 16, seed=0)}[name]()
    plan = _core.fused_plan_dump(c.model_dump_json())
    assert _plan_cost(plan) <= cost_max
    if name in ("bw30", "hea26"):
        assert max(_spread(p["qubits"]) for p in plan["passes"]) <= 24
    # every operation lands in exactly one pass
    assert sum(p["raw"] for p in plan["passes"]) == len(_core.compile_dump(c.model_dump_json()))


def _plan_in_child(text, queue):
    plan = _core.fused_plan_dump(text)
    queue.put((len(plan["passes"]), sum(len(p["blocks"]) for p in plan["passes"])))


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_planning_in_a_forked_child():
    """Planning runs on pooled host workers; a child forked after the pool
    started has none of them and plans on its calling thread, to the same plan."""
    import multiprocessing as mp

    from dqsim import workloads

    text = workloads.brickwork(24, 12, seed=2, measure=False).model_dump_json()
    plan = _core.fused_plan_dump(text)  # starts the pool in this process
    expect = (len(plan["passes"]), sum(len(p["blocks"]) for p in plan["passes"]))
    ctx = mp.get_context("fork")
    queue = ctx.Queue()
    child = ctx.Process(target=_plan_in_child, args=(text, queue))
    child.start()
    child.join(120)
    assert child.exitcode == 0
    assert queue.get(timeout=5) == expect


def warp_wavefronts(offsets, entry_bytes):
    """Shared-memory wavefronts of one warp store (one per 128 bytes, more on bank conflicts)."""
    banks = (np.asarray(offsets) // 4) % 32
    if entry_bytes == 4:
        return int(np.bincount(banks, minlength=32).max())
    # 8-byte entries go out a half-warp (128 bytes) at a time
    return sum(int(np.bincount(banks[h * 16:(h + 1) * 16] // 2, minlength=16).max()) for h in range(2))


@pytest.mark.parametrize("maker", [lambda: brickwork(30, 40, seed=0, measure=False), lambda: qft(30, seed=0),
                                   lambda: hea(26, 20, seed=0), lambda: random_circuit_n(20, 400, 5)])
def test_split_and_stage_stores_avoid_bank_conflicts(maker):
    plan = _core.fused_plan_dump(maker().model_dump_json())
    split_extra = 0
    for p in plan["passes"]:
        in_lo, in_hi = np.asarray(p["in_lo"]), np.asarray(p["in_hi"])
        pos, qoff = p["split_pos"], np.asarray(p["split_qoff"])
        # split: a warp (lanes = bits 0..4 of gt) stores one 4-byte entry per lane
        for w in range(4):
            gt = np.arange(32) + 32 * w
            P = np.zeros(32, dtype=np.int64)
            for b in range(1, 8):
                P |= (((2 * gt) >> b) & 1) << pos[b]
            off = (in_lo[P & 63] ^ in_hi[P >> 6]) ^ qoff[3]
            split_extra += warp_wavefronts(off, 4) - 1
        # stage: the last block's readback, lanes = its TMEM lanes (tile columns)
        nc = np.asarray(p["blocks"][-1]["next_c"])
        for w in range(4):
            assert warp_wavefronts(nc[32 * w:32 * w + 32], 8) == 2
        # the stage keeps the amplitudes e and e ^ 1 in one 16-byte pair
        out = np.asarray(p["out_lo"])[np.arange(4096) & 63] ^ np.asarray(p["out_hi"])[np.arange(4096) >> 6]
        assert np.all((out[0::2] ^ out[1::2]) == 8)
    # at most one conflicting warp store in ten, across the plan
    assert split_extra <= 0.1 * 4 * len(plan["passes"]), split_extra

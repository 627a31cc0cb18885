"""P-block dense blocks on the device (dq_block_*) against the CPU oracle.

The reference's P-block model (src/distributed/pblock/model.rs) runs every
gate, merge and measurement on one dense block with the src/engine.rs kernels;
these tests drive the same calls through the C ABI on device blocks and
compare them with the oracle's restatement of those kernels on the host
(amplitudes to 1e-12 in complex128, outcomes exactly), then replay P-block
style block bookkeeping -- independent Bell-pair blocks, a gate across two
blocks that merges them (model.rs:249-258), mid-circuit measurement of one
block, sampling tables per block -- and check the product of the blocks
against the statevector oracle run of the same circuit.
"""

import ctypes

import numpy as np
import pytest

from oracle import oracle as o

from dqsim import _core

pytestmark = pytest.mark.gpu
TOL = 1e-12


def dev(a):
    """A device copy, complete before it returns: the block context runs on a non-blocking stream of its own,
    which does not wait for torch's stream."""
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    torch.cuda.synchronize()
    return t


def host(t):
    return t.cpu().numpy()


def rand_state(rng, n):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def rand_unitary(rng, k):
    z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def ints(xs):
    return np.ascontiguousarray(list(xs), dtype=np.int32)


@pytest.mark.parametrize("n", [4, 5, 12, 13])
def test_block_gates_match_the_oracle(n):
    rng = np.random.default_rng(n)
    ctx = _core.BlockContext()
    L = o.lib()
    s = rand_state(rng, n)
    t = dev(s)
    want = s.copy()
    for step in range(24):
        kind = step % 5
        qs = rng.choice(n, size=min(n, 4), replace=False).tolist()
        if kind == 0:  # controlled one-qubit gate
            u = rand_unitary(rng, 1)
            ctl = [(qs[1], True), (qs[2], bool(step & 1))]
            ctx.apply_one_qubit(t.data_ptr(), n, qs[0], u, ctl)
            cq, cv = ints([c for c, _ in ctl]), ints([int(v) for _, v in ctl])
            L.orc_apply_one_qubit(P(want), n, qs[0], P(np.ascontiguousarray(u.reshape(4))), P(cq), P(cv), 2, 0, 1)
        elif kind == 1:  # controlled X
            ctx.apply_x(t.data_ptr(), n, qs[0], [(qs[1], True)])
            cq, cv = ints([qs[1]]), ints([1])
            x = np.array([0, 1, 1, 0], dtype=np.complex128)
            L.orc_apply_one_qubit(P(want), n, qs[0], P(x), P(cq), P(cv), 1, 1, 1)
        elif kind == 2:  # controlled swap
            ctx.apply_swap(t.data_ptr(), n, qs[0], qs[1], [(qs[2], True)])
            cq, cv = ints([qs[2]]), ints([1])
            L.orc_apply_swap(P(want), n, qs[0], qs[1], P(cq), P(cv), 1, 1)
        elif kind == 3:  # diagonal on three qubits
            d = np.exp(1j * rng.uniform(0, 2 * np.pi, size=8))
            ctx.apply_diagonal(t.data_ptr(), n, qs[:3], d)
            L.orc_apply_diagonal(P(want), n, P(ints(qs[:3])), 3, P(np.ascontiguousarray(d)), 1)
        else:  # dense on 2..4 qubits (DenseLayout)
            k = 2 + step % 3
            u = rand_unitary(rng, k)
            ctx.apply_dense(t.data_ptr(), n, qs[:k], u)
            L.orc_apply_dense(P(want), n, P(ints(qs[:k])), k, P(np.ascontiguousarray(u.reshape(-1))), 1)
    ctx.sync()
    assert np.max(np.abs(host(t) - want)) <= TOL


def test_merge_is_the_product_state_and_measurement_matches():
    import torch

    rng = np.random.default_rng(3)
    ctx = _core.BlockContext()
    left, right = rand_state(rng, 3), rand_state(rng, 4)
    tl, tr = dev(left), dev(right)  # kept alive until the context's stream has read them
    out = torch.empty(1 << 7, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    ctx.merge(tl.data_ptr(), 3, tr.data_ptr(), 4, out.data_ptr())
    ctx.sync()
    # model.rs:216-230: chunk i of the merged state is the left block times right[i].
    assert np.max(np.abs(host(out) - np.kron(right, left))) <= TOL
    L = o.lib()
    want = np.kron(right, left)
    for q, draw in ((0, 0.31), (6, 0.77), (3, 0.02)):
        got = ctx.measure(out.data_ptr(), 7, q, draw)
        expect = L.orc_measure(P(want), 7, q, draw, 1, None)
        assert got == expect
        assert np.max(np.abs(host(out) - want)) <= TOL


def test_probabilities_and_running_sums():
    import torch

    rng = np.random.default_rng(5)
    ctx = _core.BlockContext()
    n = 13
    s = rand_state(rng, n)
    t = dev(s)
    probs = torch.empty(1 << n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.probabilities(t.data_ptr(), n, None, probs.data_ptr())
    sums = torch.empty(1 << n, dtype=torch.float64, device="cuda")
    ctx.running_sums(t.data_ptr(), n, sums.data_ptr())
    marg = torch.empty(8, dtype=torch.float64, device="cuda")
    ctx.probabilities(t.data_ptr(), n, [9, 0, 4], marg.data_ptr())
    ctx.sync()
    p = np.abs(s) ** 2
    assert np.max(np.abs(host(probs) - p)) <= 1e-15
    assert np.max(np.abs(host(sums) - np.cumsum(p))) <= TOL  # model.rs:583-608 (running |a|^2)
    want = o.marginal_probs(s, n, [9, 0, 4])
    assert np.max(np.abs(host(marg) - want)) <= 1e-14


def test_pblock_bookkeeping_on_device_blocks_matches_the_statevector():
    """Four qubits as two Bell-pair blocks; CX(1, 2) merges them (the left block keeps the low local
    qubits, model.rs:199-248); qubit 0 is measured with a fixed draw; a CZ then runs on the merged block.
    The merged block, with its local-to-wire order undone, is the statevector oracle's state."""
    import torch

    ctx = _core.BlockContext()
    h = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
    blocks = {}
    for wires in ((0, 1), (2, 3)):
        b = torch.zeros(4, dtype=torch.complex128, device="cuda")
        b[0] = 1
        torch.cuda.synchronize()
        ctx.apply_one_qubit(b.data_ptr(), 2, 0, h)
        ctx.apply_x(b.data_ptr(), 2, 1, [(0, True)])
        blocks[wires] = b
    merged = torch.empty(16, dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    ctx.merge(blocks[(0, 1)].data_ptr(), 2, blocks[(2, 3)].data_ptr(), 2, merged.data_ptr())
    local = [0, 1, 2, 3]  # wire of each local qubit after the merge
    ctx.apply_x(merged.data_ptr(), 4, local.index(2), [(local.index(1), True)])
    outcome = ctx.measure(merged.data_ptr(), 4, local.index(0), 0.6)
    ctx.apply_diagonal(merged.data_ptr(), 4, [local.index(3), local.index(0)], [1, 1, 1, -1])
    ctx.sync()
    ops = [("one", 0, [[h[0, 0], h[0, 1]], [h[1, 0], h[1, 1]]], ()), ("x", 1, ((0, True),)),
           ("one", 2, [[h[0, 0], h[0, 1]], [h[1, 0], h[1, 1]]], ()), ("x", 3, ((2, True),)),
           ("x", 2, ((1, True),))]
    want = o.zero_state(4)
    for op in ops:
        o.apply_op(op, want, 4, [], None, True)
    expect = o.lib().orc_measure(P(want), 4, 0, 0.6, 1, None)
    o.apply_op(("diag", (3, 0), (1, 1, 1, -1)), want, 4, [], None, True)
    assert outcome == expect
    assert np.max(np.abs(host(merged) - want)) <= TOL

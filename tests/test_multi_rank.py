"""bench.py's multi-rank plumbing on CPU: two gloo ranks over 127.0.0.1 take
the same barrier and all-reduce steps as the NCCL ranks of `--gpus N` (each
rank a replica; the step time is the maximum over ranks)."""

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, str(ROOT))
    import bench

    w, r, local, pg = bench.dist_setup(None)
    assert (w, r, local) == (world, rank, rank) and pg is not None
    bench.barrier(pg)
    # rank r "took" 10 + r ms: every rank must see the slowest
    slowest = bench.max_over_ranks(pg, local, 10.0 + rank)
    bench.barrier(pg)
    out.put((rank, slowest))
    pg.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_the_slowest_step():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert got == {0: 11.0, 1: 11.0}


def test_single_rank_needs_no_process_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    sys.path.insert(0, str(ROOT))
    import bench

    world, rank, local, pg = bench.dist_setup(None)
    assert (world, rank, local, pg) == (1, 0, 0, None)
    assert bench.max_over_ranks(pg, local, 3.5) == 3.5


def test_partition_is_a_balanced_exact_cover():
    sys.path.insert(0, str(ROOT / "classical-quantum-sim-optimizer_b200"))
    from dqsim import sharding, workloads

    circuits = workloads.hea_batch(64, seed=5)
    weights = [sharding.circuit_weight(c) for c in circuits]
    for world in (1, 2, 3, 8):
        shares = sharding.partition(weights, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(circuits)))
        loads = [sum(weights[i] for i in s) for s in shares]
        # longest-processing-time bound: no rank exceeds the mean load by more than one item
        assert max(loads) <= sum(weights) / world + max(weights)
        assert shares == sharding.partition(weights, world)  # depends on the weights alone
    with pytest.raises(ValueError):
        sharding.partition(weights, 0)


def batch_rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "classical-quantum-sim-optimizer_b200"))
    import bench
    from dqsim import sharding, workloads
    from helpers import zz_expectation
    from oracle import oracle

    w, r, local, pg = bench.dist_setup(None)
    circuits = workloads.hea_batch(12, seed=3, qmin=4, qmax=8, dmin=2, dmax=5)
    mine, share = sharding.shard(circuits, w, r)
    sim = oracle.OracleSimulator(seed=11)
    zz = [zz_expectation(sim.simulate(c).statevector) for c in share]
    counts = [oracle.OracleSimulator(seed=100 + i).simulate_shots(circuits[i], shots=64) for i in mine]
    zz_all = sharding.merge_values(pg, mine, zz, len(circuits))
    counts_all = sharding.merge_counts(pg, mine, counts, len(circuits))
    out.put((r, mine, zz_all, counts_all))
    pg.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_shard_a_batch_and_merge_its_results():
    """Each rank runs its share (the oracle stands in for the device on CPU ranks);
    the all-reduce and the gather rebuild what one process computes."""
    sys.path.insert(0, str(ROOT / "classical-quantum-sim-optimizer_b200"))
    from dqsim import workloads
    from helpers import zz_expectation
    from oracle import oracle

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=batch_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, mine, zz_all, counts_all = out.get(timeout=150)
        got[r] = (mine, zz_all, counts_all)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    circuits = workloads.hea_batch(12, seed=3, qmin=4, qmax=8, dmin=2, dmax=5)
    assert sorted(got[0][0] + got[1][0]) == list(range(len(circuits))) and got[0][0] and got[1][0]
    want_zz = [zz_expectation(oracle.OracleSimulator(seed=11).simulate(c).statevector) for c in circuits]
    assert got[0][1] == got[1][1] == want_zz
    assert got[1][2] is None
    assert got[0][2] == [oracle.OracleSimulator(seed=100 + i).simulate_shots(c, shots=64)
                         for i, c in enumerate(circuits)]

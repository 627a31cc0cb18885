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

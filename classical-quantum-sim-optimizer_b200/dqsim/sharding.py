"""Batch workloads across GPUs: one process per GPU, circuits partitioned, results merged.

A batch of independent circuits (the reference's evaluation and data
collection sets, scripts/collect_simulator_data.py:104-129 runs them one by
one) shards with no data-path exchange: every rank runs its share as one
``BatchedCircuits`` graph on its own GPU.  Per-circuit scalars merge with a
single all-reduce of a dense vector, and shot histograms, which are small and
sparse, merge on the host with one gather to rank 0.  The functions take a
``torch.distributed`` module (or ``None`` for one process) so the same code
runs over NCCL on GPUs and over gloo on CPU ranks.
"""

from __future__ import annotations

import heapq


def circuit_weight(circuit):
    """Amplitude-operations of a circuit: 2^n x instructions (the cost a dense pass scales with)."""
    return (1 << int(circuit.num_qubits)) * max(1, len(circuit.data["instructions"]))


def partition(weights, world):
    """Longest-processing-time assignment of items to ``world`` ranks.

    Items go heaviest first (ties by index) to the rank with the least load so
    far (ties by rank), so the result depends only on the weights.  Returns one
    ascending index list per rank; every index appears exactly once.
    """
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(s) for s in shares]


def shard(circuits, world, rank):
    """Indices and circuits of ``rank``'s share of the batch."""
    idx = partition([circuit_weight(c) for c in circuits], world)[rank]
    return idx, [circuits[i] for i in idx]


def merge_values(dist, indices, values, total, device="cpu"):
    """Every rank's per-circuit scalars, placed by circuit index, summed over ranks (one all-reduce).

    Returns a list of ``total`` floats on every rank.  With ``dist`` None the
    local values are only placed.
    """
    import torch

    full = torch.zeros(total, dtype=torch.float64, device=device)
    if len(indices):
        full[torch.as_tensor(list(indices), dtype=torch.int64, device=device)] = torch.as_tensor(
            [float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(full, op=dist.ReduceOp.SUM)
    return full.cpu().tolist()


def merge_counts(dist, indices, counts, total):
    """Shot histograms of every rank's circuits, gathered to rank 0 in circuit order.

    Rank 0 gets a list of ``total`` dictionaries; the other ranks get None.
    """
    local = list(zip(indices, counts))
    if dist is None:
        parts = [local]
    else:
        rank = dist.get_rank()
        parts = [None] * dist.get_world_size() if rank == 0 else None
        dist.gather_object(local, parts, dst=0)
        if rank != 0:
            return None
    out = [None] * total
    for part in parts:
        for i, c in part:
            if out[i] is not None:
                raise RuntimeError(f"circuit {i} was run by two ranks")
            out[i] = c
    missing = [i for i, c in enumerate(out) if c is None]
    if missing:
        raise RuntimeError(f"circuits {missing[:8]} were run by no rank")
    return out

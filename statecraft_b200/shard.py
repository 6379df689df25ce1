"""Sharding of the batched workloads over GPUs (one process per GPU).

QAOA instances and noisy trajectories are independent, so N ranks split a batch
with no data-path collective: each rank evaluates its share on its own GPU and the
per-instance results meet on rank 0 in one host gather at the end.  A trajectory
keeps its global index, so its seeds (noise_seed + t, measure_seed + t) and hence
its outcomes do not depend on the number of ranks.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np


def partition_by_cost(costs: Sequence[float], world: int) -> list[np.ndarray]:
    """Splits item indices over `world` ranks, balancing the summed cost: items in
    decreasing cost order go to the least-loaded rank (ties to the lower rank).
    Deterministic; each rank's indices are returned in increasing order."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def contiguous_range(count: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's share of `count` equal-cost items (e.g. trajectories)."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def qaoa_costs(n_qubits: Sequence[int]) -> np.ndarray:
    """HBM work of one instance of the batched QAOA kernels: proportional to 2^n."""
    return np.exp2(np.asarray(n_qubits, dtype=np.float64))


def gather_by_index(values: np.ndarray, indices: np.ndarray, count: int, group=None):
    """Assembles per-item results from every rank on rank 0 (None elsewhere).
    `values[k]` belongs to global item `indices[k]`."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    payload = (np.asarray(indices, dtype=np.int64), np.asarray(values))
    parts = [None] * world if rank == 0 else None
    dist.gather_object(payload, parts, dst=0, group=group)
    if rank != 0:
        return None
    first = np.asarray(parts[0][1])
    out = np.zeros((count,) + first.shape[1:], dtype=first.dtype)
    seen = np.zeros(count, dtype=bool)
    for idx, val in parts:
        out[idx] = val
        seen[idx] = True
    if not seen.all():
        raise RuntimeError("gather: some items were evaluated by no rank")
    return out

"""Event sharding across ranks (one process per GPU) for the batched and serving paths.

Events are independent, so ranks never exchange point data: every rank clusters the events
assigned to it and only the per-event results travel back to the gathering rank, over the
host (torch.distributed object collectives; gloo on CPU, NCCL-backed groups on GPUs).
The single-event path does not shard (its candidate searches cross any spatial cut) and runs
as replicas.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition_events(sizes, world: int) -> list[np.ndarray]:
    """Assigns events to `world` ranks, balancing the points per rank: events are taken
    largest first and each goes to the rank with the fewest points so far (ties: lowest rank).
    Returns, per rank, its event ids in ascending order.  Deterministic."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    owner = np.empty(sizes.size, np.int64)
    for e in np.argsort(-sizes, kind="stable"):
        load, r = heapq.heappop(heap)
        owner[e] = r
        heapq.heappush(heap, (load + int(sizes[e]), r))
    return [np.nonzero(owner == r)[0] for r in range(world)]


def gather_event_results(local: dict, world: int, rank: int, dst: int = 0):
    """Gathers {event id: per-event result} dicts from every rank onto `dst` (None elsewhere).
    Uses torch.distributed's object gather, so it works with gloo and NCCL groups alike."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    bucket = [None] * world if rank == dst else None
    dist.gather_object(local, bucket, dst=dst)
    if rank != dst:
        return None
    merged = {}
    for part in bucket:
        dup = merged.keys() & part.keys()
        if dup:
            raise RuntimeError(f"events {sorted(dup)[:5]} returned by two ranks")
        merged.update(part)
    return merged

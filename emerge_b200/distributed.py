"""Frequency-partitioned sweeps across GPUs (one process per GPU).

The sweep has no exchange step: every (frequency, port) system is independent and every rank can
assemble its own E/B (milliseconds).  Systems are dealt round-robin by cost order, each rank solves
its share on its own GPU, and the per-system results (status, iterations, FP64 relative residual,
optional extracted quantities) are gathered on the host with one object all-gather.  This mirrors
the reference's frequency-parallel run_sweep (threads/processes, ``MW/microwave_3d.py:795-861``).
"""
from __future__ import annotations

from typing import Callable, Sequence


def partition(systems: Sequence, world_size: int, rank: int) -> list[tuple[int, object]]:
    """Round-robin share of ``systems`` for ``rank`` as (global index, system) pairs."""
    if world_size < 1 or not (0 <= rank < world_size):
        raise ValueError(f"bad rank {rank} for world size {world_size}")
    return [(i, s) for i, s in enumerate(systems) if i % world_size == rank]


def gather(local: list[tuple[int, object]], n_total: int) -> list:
    """All-gather (index, result) pairs from every rank and return results in global order."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        parts: list = [None] * dist.get_world_size()
        dist.all_gather_object(parts, local)
        merged = [p for part in parts for p in part]
    else:
        merged = list(local)
    out: list = [None] * n_total
    for i, r in merged:
        if out[i] is not None:
            raise RuntimeError(f"system {i} solved twice")
        out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"systems {missing[:8]} were not solved by any rank")
    return out


def run_partitioned(systems: Sequence, solve_batch: Callable[[list], list], world_size: int, rank: int,
                    batch: int = 64) -> list:
    """Solve this rank's share in batches of <= ``batch`` with ``solve_batch(list_of_systems) ->
    list_of_results`` and gather all results in global order."""
    mine = partition(systems, world_size, rank)
    local = []
    for b0 in range(0, len(mine), batch):
        chunk = mine[b0:b0 + batch]
        res = solve_batch([s for _, s in chunk])
        local.extend((i, r) for (i, _), r in zip(chunk, res))
    return gather(local, len(systems))

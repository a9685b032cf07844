"""Frequency-partitioned sweeps across GPUs (one process per GPU).

The sweep has no exchange step: every (mesh, frequency, port) system is independent and every rank
assembles its own E/B (milliseconds).  Work items are dealt by a cost model: sorted by decreasing cost
and each given to the rank with the least total cost so far (longest-processing-time first, ties to the
lower rank), so uneven meshes balance across GPUs.  Each rank solves its share on its own GPU, and the
per-item results (status, iterations, FP64 relative residual, extracted quantities) are gathered on the
host with one object all-gather.  This mirrors the reference's frequency-parallel run_sweep
(threads/processes, ``MW/microwave_3d.py:795-861``), which hands frequencies to workers in order.
"""
from __future__ import annotations

from typing import Callable, Sequence


def partition(systems: Sequence, world_size: int, rank: int, cost: Sequence[float] | None = None
              ) -> list[tuple[int, object]]:
    """This rank's share of ``systems`` as (global index, system) pairs, in ascending index order.

    ``cost`` (one number per system, e.g. the DOFs of its mesh times its Krylov work) balances the
    total cost per rank greedily; without it every system costs the same and the deal is round-robin."""
    if world_size < 1 or not (0 <= rank < world_size):
        raise ValueError(f"bad rank {rank} for world size {world_size}")
    n = len(systems)
    if cost is None:
        return [(i, s) for i, s in enumerate(systems) if i % world_size == rank]
    if len(cost) != n:
        raise ValueError("one cost per system")
    order = sorted(range(n), key=lambda i: (-float(cost[i]), i))
    load = [0.0] * world_size
    owner = [0] * n
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += float(cost[i])
    return [(i, systems[i]) for i in range(n) if owner[i] == rank]


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
                    batch: int = 64, cost: Sequence[float] | None = None) -> list:
    """Solve this rank's share in batches of <= ``batch`` with ``solve_batch(list_of_systems) ->
    list_of_results`` and gather all results in global order."""
    mine = partition(systems, world_size, rank, cost)
    local = []
    for b0 in range(0, len(mine), batch):
        chunk = mine[b0:b0 + batch]
        res = solve_batch([s for _, s in chunk])
        local.extend((i, r) for (i, _), r in zip(chunk, res))
    return gather(local, len(systems))


def world() -> tuple[int, int]:
    """(world_size, rank) of the initialised process group, (1, 0) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0

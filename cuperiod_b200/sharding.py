"""Curve-parallel searches over the GPUs of one node: one process per GPU
(launched by torchrun), each searching its own shard of the light curves.

Light curves are independent (the reference searches each on its own,
src/cuperiod/batch/runner.py:214-250, and every trial period of a curve on its
own, src/cuperiod/methods/_bls_core.py:356), so the data path has no collective.
A rank's shard is chosen by cost, points x trial periods, with a longest-first
greedy assignment.  Only the per-curve result rows travel, gathered to rank 0
once at the end; step timings are combined as the maximum over ranks.
"""

from __future__ import annotations

from typing import Any, Callable, Sequence

from .batch import BatchSummary, batch_periodograms


def _dist():
    import torch.distributed as dist
    return dist


def world_info(group: Any = None) -> tuple[int, int]:
    """(rank, world size) of the default process group, or (0, 1) without one."""
    dist = _dist()
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def shard_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of each rank's shard: the costliest item first, each to the rank
    with the least cost so far (ties to the lower rank), each shard in input
    order.  Deterministic, so every rank computes the same partition alone."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        shards[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(s) for s in shards]


def _n_points(data: Any) -> int:
    if hasattr(data, "t"):
        return int(len(data.t))
    return int(len(data[0]))


def max_over_ranks(x: float, group: Any = None) -> float:
    """The largest of every rank's ``x`` (a step time): a one-element all-reduce,
    on the GPU for NCCL groups and on the host for gloo."""
    rank, world = world_info(group)
    if world == 1:
        return float(x)
    import torch
    dist = _dist()
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def batch_periodograms_sharded(inputs: Sequence[tuple[str, Any]], method: str = "BLS", *,
                               group: Any = None, sink: str | None = None,
                               runner: Callable[..., BatchSummary] = batch_periodograms,
                               **kwargs: Any) -> BatchSummary | None:
    """``batch_periodograms`` over this rank's shard of ``inputs``; rank 0 gathers
    every rank's rows and errors and returns them in input order (and writes
    ``sink``), the other ranks return None.  Every rank must pass the same
    ``inputs``.  With no process group this is ``batch_periodograms`` itself.
    ``runner`` is the per-shard search (the default engine path)."""
    inputs = list(inputs)
    rank, world = world_info(group)
    if world == 1:
        return runner(inputs, method, sink=sink, **kwargs)
    shards = shard_by_cost([_n_points(d) for _, d in inputs], world)
    local = runner([inputs[i] for i in shards[rank]], method, **kwargs)
    payload = (local.rows, local.errors, local.launches)
    dist = _dist()
    gathered: list | None = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    position: dict[str, int] = {}
    for i, (key, _) in enumerate(inputs):
        position.setdefault(str(key), i)
    summary = BatchSummary()
    for rows, errors, launches in gathered:
        summary.rows.extend(rows)
        summary.errors.update(errors)
        summary.launches += launches
    summary.rows.sort(key=lambda row: position.get(str(row["key"]), len(inputs)))
    if sink is not None and summary.rows:
        import pyarrow as pa
        import pyarrow.parquet as pq
        pq.write_table(pa.Table.from_pylist(summary.rows), sink)
    return summary


__all__ = ["batch_periodograms_sharded", "max_over_ranks", "shard_by_cost", "world_info"]

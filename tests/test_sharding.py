"""Curve sharding across ranks: the partition on its own, and two gloo ranks on the
host running the sharded batch entry and the max-over-ranks timing helper."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from cuperiod_b200.batch import BatchSummary
from cuperiod_b200.sharding import batch_periodograms_sharded, max_over_ranks, shard_by_cost


def test_shard_by_cost_partitions_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.integers(500, 20000, size=101).tolist()
    for world in (1, 2, 3, 8):
        shards = shard_by_cost(costs, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        for s in shards:
            assert s == sorted(s)
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)
    assert shard_by_cost(costs, 4) == shard_by_cost(costs, 4)
    with pytest.raises(ValueError):
        shard_by_cost(costs, 0)


def test_single_process_is_the_plain_batch():
    seen = {}

    def runner(inputs, method, sink=None, **kw):
        seen["n"] = len(inputs)
        return BatchSummary(rows=[{"key": k} for k, _ in inputs])

    out = batch_periodograms_sharded([("a", ([0, 1], [1, 1])), ("b", ([0], [1]))], runner=runner)
    assert seen["n"] == 2 and [r["key"] for r in out.rows] == ["a", "b"]


def _fake_runner(inputs, method, **kw):
    """Stands in for the engine: one row per curve carrying its point count and
    the rank that searched it; curves of one point fail."""
    import torch.distributed as dist
    s = BatchSummary(launches=1)
    for key, (t, y) in inputs:
        if len(t) < 2:
            s.errors[key] = "InsufficientDataError"
        else:
            s.rows.append({"key": key, "n": len(t), "rank": dist.get_rank()})
    return s


def _inputs():
    sizes = [7, 1, 30, 12, 5, 5, 18, 2, 40, 9, 1, 22]
    return [(f"c{i}", (list(range(n)), [1.0] * n)) for i, n in enumerate(sizes)]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    from datetime import timedelta

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = batch_periodograms_sharded(_inputs(), runner=_fake_runner)
        m = max_over_ranks(10.0 + rank)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            if res is None:
                f.write(f"none {m}\n")
            else:
                f.write(f"rows {m} {res.launches} {len(res.errors)}\n")
                for row in res.rows:
                    f.write(f"{row['key']} {row['n']} {row['rank']}\n")
                f.write("errors " + " ".join(sorted(res.errors)) + "\n")
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_gather(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r1 = (tmp_path / "rank1.txt").read_text().split()
    assert r1[0] == "none" and float(r1[1]) == 11.0
    lines = (tmp_path / "rank0.txt").read_text().splitlines()
    head = lines[0].split()
    assert head[0] == "rows" and float(head[1]) == 11.0      # max over ranks
    assert int(head[2]) == world                             # one launch per rank
    rows = [ln.split() for ln in lines[1:-1]]
    expected = [k for k, (t, _) in _inputs() if len(t) >= 2]
    assert [r[0] for r in rows] == expected                  # input order restored
    by_rank = {0: 0, 1: 0}
    for key, n, rank in rows:
        by_rank[int(rank)] += int(n)
    assert by_rank[0] > 0 and by_rank[1] > 0                 # both ranks searched
    assert lines[-1].split()[1:] == ["c1", "c10"]           # errors gathered

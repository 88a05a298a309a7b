"""The tile-shape autotuner's host logic with a fake clock (no device)."""

from __future__ import annotations

import json

import numpy as np
import pytest


def _batch(n=40, seed=3):
    from cuperiod_b200 import _lib
    rng = np.random.default_rng(seed)
    curves = []
    for _ in range(n):
        m = int(rng.integers(50, 400))
        t = np.sort(rng.uniform(0.0, 30.0, m))
        curves.append((t, 1.0 + 1e-3 * rng.normal(size=m), None))
    grid = _lib.PackedGrid.from_segments(
        [(np.geomspace(0.5, 1.0, 50), np.array([0.02, 0.04])),
         (np.geomspace(1.0, 2.0, 30)[1:], np.array([0.04, 0.08]))], 10, 0)
    return grid, _lib.PackedCurves.from_arrays(curves)


def test_sample_spans_the_length_order():
    from cuperiod_b200.autotune import sample_indices
    n = np.array([5, 100, 7, 50, 3, 900, 20, 8])
    idx = sample_indices(n, 3)
    assert list(idx) == sorted(idx)
    lens = sorted(n[idx])
    assert lens[0] == 3 and lens[-1] == 900           # shortest and longest kept
    assert list(sample_indices(n, 20)) == list(range(8))


def test_subset_repacks_the_chosen_curves():
    from cuperiod_b200.autotune import subset
    _, curves = _batch(6)
    sub = subset(curves, [1, 4])
    off = curves.offsets
    assert sub.n_curves == 2
    np.testing.assert_array_equal(sub.t[:sub.offsets[1]], curves.t[off[1]:off[2]])
    np.testing.assert_array_equal(sub.y[sub.offsets[1]:], curves.y[off[4]:off[5]])


def test_picks_the_fastest_and_records_failures(tmp_path):
    from cuperiod_b200.autotune import TileShape, autotune
    from cuperiod_b200.errors import BackendUnavailableError
    grid, curves = _batch()
    clock = {TileShape(0, 0): 10.0, TileShape(0, 4): 7.5, TileShape(0, 8): 9.0}
    seen = []

    def timer(shape, g, sample):
        seen.append((shape, sample.n_curves))
        if shape.smem_per_cta == 200 * 1024:
            raise BackendUnavailableError("too wide")
        return clock[shape]

    cands = [TileShape(0, 0), TileShape(0, 8), TileShape(0, 4), TileShape(0, 8),
             TileShape(200 * 1024, 0)]
    cache = tmp_path / "tune.json"
    res = autotune(grid, curves, candidates=cands, sample=16, timer=timer, cache=cache,
                   refresh=True)
    assert res.shape == TileShape(0, 4) and not res.cached
    assert [s for s, _ in seen] == [TileShape(0, 0), TileShape(0, 8), TileShape(0, 4),
                                    TileShape(200 * 1024, 0)]     # repeats timed once
    assert all(n == 16 for _, n in seen)
    assert res.ms == {"smem=default,tile=fit": 10.0, "smem=default,tile=8": 9.0,
                      "smem=default,tile=4": 7.5}
    assert list(res.errors) == ["smem=200K,tile=fit"]
    assert res.speedup_over_default() == pytest.approx(10.0 / 7.5)
    # memory, then file, caches answer without timing
    seen.clear()
    again = autotune(grid, curves, candidates=cands, sample=16, timer=timer)
    assert again.cached and again.shape == res.shape and not seen
    from cuperiod_b200 import autotune as mod
    mod._memory.clear()
    row = json.loads(cache.read_text())[res.key]
    assert (row["smem_per_cta"], row["max_tile"]) == (0, 4)
    from_file = autotune(grid, curves, candidates=cands, sample=16, timer=timer, cache=cache)
    assert from_file.cached and from_file.shape == TileShape(0, 4) and not seen


def test_no_runnable_shape_is_an_error():
    from cuperiod_b200.autotune import TileShape, autotune
    from cuperiod_b200.errors import BackendUnavailableError
    grid, curves = _batch(4)

    def timer(shape, g, sample):
        raise BackendUnavailableError("does not fit")

    with pytest.raises(BackendUnavailableError, match="no candidate shape"):
        autotune(grid, curves, candidates=[TileShape(0, 0)], timer=timer, refresh=True)
    with pytest.raises(ValueError):
        autotune(grid, curves, candidates=[], timer=timer)


def test_key_separates_workloads():
    from cuperiod_b200 import _lib
    from cuperiod_b200.autotune import workload_key
    grid, curves = _batch()
    k = workload_key(grid, curves, "B200")
    assert k == workload_key(grid, curves, "B200")
    assert k != workload_key(grid, curves, "other")
    ll = _lib.PackedGrid(grid.seg_offsets, grid.periods, grid.dur_offsets, grid.durations,
                         grid.oversample, 1)
    assert k != workload_key(ll, curves, "B200")
    dy = _lib.PackedCurves(curves.offsets, curves.t, curves.y,
                           np.linspace(1.0, 2.0, curves.t.size))
    assert k != workload_key(grid, dy, "B200")


def test_a_corrupt_cache_file_is_ignored(tmp_path):
    from cuperiod_b200 import autotune as mod
    from cuperiod_b200.autotune import TileShape, autotune
    grid, curves = _batch(6)
    cache = tmp_path / "tune.json"
    cache.write_text("{not json")
    mod._memory.clear()
    res = autotune(grid, curves, candidates=[TileShape(0, 0), TileShape(0, 4)],
                   timer=lambda shape, g, s: 2.0 if shape.max_tile else 3.0, cache=cache)
    assert res.shape == TileShape(0, 4) and not res.cached
    assert json.loads(cache.read_text())[res.key]["max_tile"] == 4    # rewritten whole

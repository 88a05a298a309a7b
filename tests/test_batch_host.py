"""batch_periodograms' host orchestration with the device step replaced by a
fake (no device): chunks, input order, failures, and which path a curve takes."""

from __future__ import annotations

import numpy as np
import pytest


def _curves(n, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        span = rng.uniform(8.0, 30.0)
        t = np.sort(rng.uniform(0.0, span, int(rng.integers(60, 400))))
        out.append((f"k{i}", (t, 1.0 + 1e-3 * rng.normal(size=t.size))))
    return out


@pytest.fixture
def fake_rows(monkeypatch):
    from cuperiod_b200.bls import BLSMethod
    calls = []

    def rows_default(self, keyed, settings, *, n_best=10, extra_keys=(), engine=None,
                     prefiltered=False):
        calls.append(("default", [k for k, _ in keyed]))
        return [{"key": k, "n": lc.n} for k, lc in keyed]

    def rows_by_grid(self, items, settings, *, n_best=10, extra_keys=(), engine=None,
                     prefiltered=False):
        calls.append(("grid", [k for k, _, _ in items]))
        return [{"key": k, "n": lc.n} for k, lc, _ in items]

    monkeypatch.setattr(BLSMethod, "rows_default", rows_default)
    monkeypatch.setattr(BLSMethod, "rows_by_grid", rows_by_grid)
    return calls


def test_default_grids_run_in_input_order_chunks(fake_rows):
    from cuperiod_b200.batch import batch_periodograms
    inputs = _curves(11)
    res = batch_periodograms(inputs, "BLS", domain="flux", chunk_size=4, workers=3)
    assert [r["key"] for r in res.rows] == [k for k, _ in inputs]
    assert res.launches == 3 and not res.errors
    assert sorted(len(keys) for kind, keys in fake_rows) == [3, 4, 4]
    assert {kind for kind, _ in fake_rows} == {"default"}


def test_failures_are_recorded_and_skipped(fake_rows):
    from cuperiod_b200.batch import batch_periodograms
    inputs = _curves(4)
    few = ("few", (np.arange(5.0), np.ones(5)))                      # < min_detections
    short = ("short", (np.linspace(0.0, 0.3, 40), np.ones(40)))      # baseline too short
    huge = ("huge", (np.array([0.0] + [1.0] * 20 + [1.0e7]), np.ones(22)))   # grid too large
    res = batch_periodograms(inputs[:2] + [few, short, huge] + inputs[2:], "BLS",
                             domain="flux")
    assert [r["key"] for r in res.rows] == [k for k, _ in inputs]
    assert set(res.errors) == {"few", "short", "huge"}
    assert res.errors["few"].startswith("InsufficientDataError")
    assert res.errors["short"].startswith("InsufficientDataError")
    assert res.errors["huge"].startswith("GridTooLargeError")


def test_an_explicit_grid_takes_the_grid_path(fake_rows):
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.grid import GridSpec
    grid = GridSpec(kind="period", values=np.geomspace(0.5, 5.0, 200))
    res = batch_periodograms(_curves(5), "BLS", domain="flux", grid=grid, chunk_size=2,
                             workers=1)
    assert [kind for kind, _ in fake_rows] == ["grid", "grid", "grid"]
    assert res.launches == 3 and len(res.rows) == 5


def test_worker_threads_persist_between_calls(monkeypatch):
    # each worker thread keeps its engine from one call to the next: the pool's
    # threads are the same ones in a second call
    import threading

    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.bls import BLSMethod
    seen = []

    def rows_default(self, keyed, settings, *, n_best=10, extra_keys=(), engine=None,
                     prefiltered=False):
        seen.append(threading.get_ident())
        return [{"key": k} for k, _ in keyed]

    monkeypatch.setattr(BLSMethod, "rows_default", rows_default)
    inputs = _curves(8)
    batch_periodograms(inputs, "BLS", domain="flux", chunk_size=2, workers=2)
    first = set(seen)
    seen.clear()
    batch_periodograms(inputs, "BLS", domain="flux", chunk_size=2, workers=2)
    assert set(seen) <= first and threading.get_ident() not in first


def test_release_workers_ends_the_pool_threads(monkeypatch):
    import threading

    from cuperiod_b200.batch import batch_periodograms, release_workers
    from cuperiod_b200.bls import BLSMethod

    def rows_default(self, keyed, settings, *, n_best=10, extra_keys=(), engine=None,
                     prefiltered=False):
        return [{"key": k} for k, _ in keyed]

    monkeypatch.setattr(BLSMethod, "rows_default", rows_default)
    batch_periodograms(_curves(6), "BLS", domain="flux", chunk_size=2, workers=3)
    assert any(t.name.startswith("bls-batch-3") for t in threading.enumerate())
    release_workers()
    assert not any(t.name.startswith("bls-batch-") for t in threading.enumerate())
    res = batch_periodograms(_curves(6), "BLS", domain="flux", chunk_size=2, workers=3)
    assert len(res.rows) == 6
    release_workers()

"""Host-side logic of the learned-pruned search (no device work): the class
edges of the log-period grid, the widened windows of a curve's top classes, and
the window grids built for many curves at once, checked against the same
windows built one curve at a time."""

from __future__ import annotations

import numpy as np

from cuperiod_b200.proposal import N_CLASSES, Proposer, class_edges, labels_of, window_mask
from cuperiod_b200.proposal_train import grid_segments


def _proposer(widen=1):
    p = Proposer.__new__(Proposer)
    p._init_grid(grid_segments(), 10, 0, widen)
    return p


def test_class_edges_cover_the_grid():
    e = class_edges(50_000)
    assert e[0] == 0 and e[-1] == 50_000 and e.size == N_CLASSES + 1
    assert np.all(np.diff(e) > 0)
    lab = labels_of(np.array([0, 49_999, 12_345]), 50_000)
    for i, c in zip((0, 49_999, 12_345), lab):
        assert e[c] <= i < e[c + 1]


def test_window_mask_widens_and_merges():
    e = class_edges(50_000)
    spans = window_mask(np.array([5, 6, 1023, 0]), e, 1)
    # classes 4..7 merge into one run; 0..1 and 1022..1023 clip at the grid's ends
    assert spans == sorted(spans)
    covered = np.zeros(50_000, bool)
    for lo, hi in spans:
        covered[lo:hi] = True
    want = np.zeros(50_000, bool)
    for c in (0, 1, 4, 5, 6, 7, 1022, 1023):
        want[e[c]:e[c + 1]] = True
    np.testing.assert_array_equal(covered, want)


def test_window_grids_match_the_per_curve_windows():
    p = _proposer()
    rng = np.random.default_rng(0)
    idx = rng.integers(0, N_CLASSES, (257, 16))
    idx[0] = 0
    idx[1] = N_CLASSES - 1
    idx[2] = np.arange(16) * 64          # classes in every segment
    grids, index = p.window_grids(idx)
    assert len(grids) == idx.shape[0]
    off = 0
    for i, g in enumerate(grids):
        spans = window_mask(idx[i], p.edges, p.widen)
        ref = np.concatenate([np.arange(lo, hi) for lo, hi in spans])
        np.testing.assert_array_equal(index[off:off + g.n_periods], ref)
        np.testing.assert_array_equal(g.periods, p.periods[ref])
        off += g.n_periods
        # each non-empty segment is the loop form's, with the full grid's durations
        segs = [g.periods[g.seg_offsets[s]:g.seg_offsets[s + 1]]
                for s in range(len(p.segments))]
        loop = p.window_segments(idx[i])
        assert [s.size for s in segs if s.size] == [q.size for q, _ in loop]
        for s, (q, _) in zip([s for s in segs if s.size], loop):
            np.testing.assert_array_equal(s, q)
        np.testing.assert_array_equal(g.durations, p.full.durations)
        np.testing.assert_array_equal(g.dur_offsets, p.full.dur_offsets)
    assert off == index.size


def test_window_grids_of_no_curves():
    grids, index = _proposer().window_grids(np.empty((0, 16), dtype=np.int64))
    assert grids == [] and index.size == 0


def test_windows_hold_is_the_window_test():
    from cuperiod_b200.proposal import windows_hold
    e = class_edges(50_000)
    rng = np.random.default_rng(3)
    idx = rng.integers(0, N_CLASSES, (500, 16))
    best = rng.integers(0, 50_000, 500)
    best[:16] = e[idx[:16, 0]]                 # on a class's first index
    best[16:32] = e[idx[16:32, 0] + 1] - 1     # on its last
    got = windows_hold(idx, best, e, 1)
    want = [any(lo <= b < hi for lo, hi in window_mask(r, e, 1)) for r, b in zip(idx, best)]
    np.testing.assert_array_equal(got, want)
    assert got[:32].all()

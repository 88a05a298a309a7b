"""The learned-pruned search returns the full search's result wherever it
searches: a window is searched with the full grid's durations for each
period's segment, so the power at every searched period equals the full
search's there, and a curve whose full-grid best period lies inside its
windows gets that period.  Below the threshold a curve is searched over the
full grid.  Checked with an untrained network (any windows will do) on curves of
the batched workload, against one plain search of the same batch; and the
streamed catalogue sweep (two workers, pinned chunks) against plain searches."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    from cuperiod_b200 import _lib
    from cuperiod_b200.proposal import Weights
    from cuperiod_b200.proposal_train import grid_segments
    from cuperiod_b200.synthetic import batched_curves
    segments = grid_segments()
    curves = [(c.t, c.y, None) for c in batched_curves(48, seed=77, n_range=(500, 4000))]
    eng = _lib.Engine()
    full = _lib.PackedGrid.from_segments(segments, 10, 0)
    eng.prepare(full, _lib.PackedCurves.from_arrays(curves))
    eng.launch()
    spectra = eng.download()[0]                  # power, (curves, periods)
    best = eng.download_best()[0]
    yield eng, segments, curves, spectra, best, Weights.init(seed=5)
    eng.close()


def test_windows_reproduce_the_full_search(setup):
    from cuperiod_b200.proposal import Proposer, window_mask
    eng, segments, curves, spectra, best, w = setup
    prop = Proposer(w, segments, threshold=0.0)          # every curve pruned
    res = prop.search(curves, eng)
    assert res.confident.all()
    for i in range(len(curves)):
        # the power the pruned search reports is the full spectrum's at that period
        assert res.best_power[i] == spectra[i, res.best_index[i]]
        classes = prop.propose([curves[i]])[0][0]
        inside = any(lo <= best[i] < hi for lo, hi in window_mask(classes, prop.edges, prop.widen))
        if inside:
            assert res.best_index[i] == best[i]
        else:
            assert res.best_power[i] <= spectra[i, best[i]]


def test_below_the_threshold_the_full_grid_is_searched(setup):
    from cuperiod_b200.proposal import Proposer
    eng, segments, curves, spectra, best, w = setup
    prop = Proposer(w, segments, threshold=2.0)          # nobody is confident
    res = prop.search(curves, eng)
    assert not res.confident.any()
    np.testing.assert_array_equal(res.best_index, best)
    assert res.periods_searched == len(curves) * sum(p.size for p, _ in segments)


def test_catalogue_sweep_matches_plain_searches(setup):
    from cuperiod_b200.catalogue import pin, sweep
    from cuperiod_b200.synthetic import catalogue_curves
    eng, segments, _, _, _, w = setup
    t, y, off, _ = catalogue_curves(600, seed=3)
    t, y, keep = pin(t, y)
    plain = sweep(t, y, off, w, segments, chunk=128, workers=2, plain=True)
    # everyone falls back: identical to the plain sweep, and every chunk was done
    fb = sweep(t, y, off, w, segments, chunk=128, workers=2, threshold=2.0)
    np.testing.assert_array_equal(fb.best_index, plain.best_index)
    assert sorted(r["chunk"] for r in fb.chunks) == list(range(5))
    # everyone pruned and audited: the audit compares with the full grid
    pr = sweep(t, y, off, w, segments, chunk=128, workers=2, threshold=0.0, audit_frac=1.0)
    assert pr.audited.all()
    np.testing.assert_array_equal(pr.audit_agree, pr.best_index == plain.best_index)
    del keep

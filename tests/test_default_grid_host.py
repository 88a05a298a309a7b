"""The engine library's default-grid builder (host code, no device) against the
Python restatement of the reference's default grid (methods/bls.py:52-125):
the same segments and the same periods bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

SETTINGS = [
    {},
    {"grid_oversample": 3},
    {"segment_factor": 1.5, "min_period_days": 0.05},
    {"max_period_days": 10.0, "min_transits": 3, "grid_duration_frac": 0.02},
    {"min_period_days": 0.3, "segment_factor": 3.0, "grid_oversample": 1},
    {"duration_min_frac": 0.02, "n_durations": 5, "min_duration_days": 0.02},
]


def _baselines(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = np.concatenate([10.0 ** rng.uniform(-0.3, 2.6, n),
                        [0.41, 0.8, 1.6, 2.0, 27.0, 90.0, 365.25, 1461.0]])
    return b


@pytest.mark.parametrize("case", range(len(SETTINGS)))
def test_periods_and_segments_are_the_references(case):
    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import _segment_durations, _segment_periods, default_grid_spec
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings(**SETTINGS[case])
    baselines = _baselines(case, 30)
    spec = default_grid_spec(s, float(baselines.max()))
    sizes = _lib.default_grid_sizes(spec, baselines)
    for b, size in zip(baselines, sizes):
        parts = _segment_periods(float(b), s)
        periods, offs, starts = _lib.default_grid(spec, float(b))
        assert size == periods.size == sum(p.size for _, p in parts)
        assert len(starts) == len(parts)
        for k, (p_lo, ref) in enumerate(parts):
            got = periods[offs[k]:offs[k + 1]]
            assert got.dtype == ref.dtype and np.array_equal(got, ref), (b, k)
            d0, d1 = spec.dur_offsets[starts[k]], spec.dur_offsets[starts[k] + 1]
            np.testing.assert_array_equal(spec.durations[d0:d1], _segment_durations(p_lo, s))


def test_default_grid_of_a_light_curve():
    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import BLSMethod, default_grid_spec
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import BLSSettings
    rng = np.random.default_rng(4)
    t = np.sort(rng.uniform(0.0, 33.3, 800)) + 2457000.0
    lc = LightCurve(t, 1.0 + 1e-3 * rng.normal(size=t.size), None, Domain.FLUX)
    s = BLSSettings()
    g = BLSMethod().default_grid(lc, s)
    periods, offs, _ = _lib.default_grid(default_grid_spec(s, lc.baseline), lc.baseline)
    assert np.array_equal(periods, g.period)
    assert list(np.diff(offs)) == list(g.meta["segment_sizes"])


def test_short_and_bad_baselines():
    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import default_grid_spec
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    spec = default_grid_spec(s, 10.0)
    # below 2 * min_period no segment starts; a bad baseline builds nothing
    assert list(_lib.default_grid_sizes(spec, [0.3, 0.0, -1.0, float("nan")])) == [0, -1, -1, -1]
    with pytest.raises(ValueError):
        _lib.default_grid(spec, 0.0)
    # a baseline past the duration table's starts is refused, not truncated
    assert _lib.default_grid_sizes(spec, [1000.0])[0] == -1


def test_split_default_records_the_references_failures():
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    short = LightCurve(np.array([0.0, 0.2, 0.3]), np.ones(3), None, Domain.FLUX)
    ok = LightCurve(np.linspace(0.0, 12.0, 50), np.ones(50), None, Domain.FLUX)
    huge = LightCurve(np.array([0.0, 1.0e7]), np.ones(2), None, Domain.FLUX)
    good, errors = BLSMethod().split_default([("s", short), ("o", ok), ("h", huge)], s)
    assert [k for k, _ in good] == ["o"]
    assert errors["s"].startswith("InsufficientDataError")
    assert errors["h"].startswith("GridTooLargeError")


def test_a_grid_beyond_the_reference_limit_is_refused_not_allocated():
    # a baseline whose default grid exceeds the reference's 250,000,000 trial
    # samples is refused before anything is allocated (1e7 days: ~2e9 periods)
    import time

    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import default_grid_spec
    from cuperiod_b200.errors import BackendUnavailableError
    from cuperiod_b200.settings import BLSSettings
    spec = default_grid_spec(BLSSettings(), 1.0e7)
    t0 = time.perf_counter()
    assert _lib.default_grid_sizes(spec, [1.0e7])[0] == -1
    with pytest.raises(BackendUnavailableError, match="250,000,000"):
        _lib.default_grid(spec, 1.0e7)
    assert time.perf_counter() - t0 < 5.0

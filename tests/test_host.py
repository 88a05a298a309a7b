"""Host-side logic of the product package against the reference's golden values:
default grids, segmentation, duration bins, peak selection and batch rows.  No
GPU is used."""

from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from _cases import GOLDEN

import cuperiod_b200 as cb
from cuperiod_b200 import bls as blsmod
from cuperiod_b200.batch import periodogram_to_row
from cuperiod_b200.core import _duration_bins
from cuperiod_b200.result import Periodogram


def test_settings_defaults_match_reference():
    s = cb.BLSSettings()
    assert (s.min_period_days, s.max_period_days, s.min_transits) == (0.2, 100.0, 2)
    assert (s.duration_min_frac, s.duration_max_frac, s.n_durations) == (0.01, 0.12, 8)
    assert (s.segment_factor, s.grid_duration_frac, s.grid_oversample) == (2.0, 0.05, 2)
    assert (s.bins_per_duration, s.objective, s.min_detections) == (10, "snr", 20)
    with pytest.raises(ValueError):
        cb.BLSSettings(min_period_days=5.0, max_period_days=1.0)


def test_settings_environment_override(monkeypatch):
    monkeypatch.setenv("CUPERIOD_BLS_N_DURATIONS", "12")
    assert cb.BLSSettings().n_durations == 12


def test_duration_bins_round_half_away_from_zero():
    assert _duration_bins(np.array([0.2, 0.25, 0.45]), 0.1) == [2, 3, 5]


GRIDS = json.load(open(os.path.join(GOLDEN, "grid_cases.json")))


@pytest.mark.parametrize("case", [g for g in GRIDS if "baseline_input" in g],
                         ids=lambda g: f"{g['baseline_input'][1] - g['baseline_input'][0]:.2f}d")
def test_default_grid_matches_reference(case):
    t0, t1, n = case["baseline_input"]
    t = np.linspace(t0, t1, n)
    lc = cb.LightCurve.from_arrays(t, np.ones(n), np.ones(n), domain="flux")
    grid = cb.BLSMethod().default_grid(lc, cb.BLSSettings(**case["settings"]))
    per = np.ascontiguousarray(grid.period, dtype=np.float64)
    assert per.size == case["size"]
    assert list(grid.meta["segment_starts"]) == case["segment_starts"]
    assert list(grid.meta["segment_sizes"]) == case["segment_sizes"]
    assert hashlib.sha256(per.tobytes()).hexdigest() == case["sha256"]


def test_log_grid_segments_match_reference():
    case = next(g for g in GRIDS if "log_grid" in g)
    lo, hi, n = case["log_grid"]
    segs = blsmod._grid_segments(cb.GridSpec(kind="period", values=np.geomspace(lo, hi, n)),
                                 cb.BLSSettings())
    assert [p.size for p, _ in segs] == case["segment_sizes"]
    for (_, d), ref in zip(segs, case["segment_durations"]):
        np.testing.assert_array_equal(d, np.asarray(ref))


def test_grid_guards():
    t = np.linspace(0.0, 200.0, 200) + 2458000.0
    t[0] = 0.0
    lc = cb.LightCurve.from_arrays(t, np.ones(t.size), np.ones(t.size), domain="flux")
    with pytest.raises(cb.GridTooLargeError):
        cb.BLSMethod().default_grid(lc, cb.BLSSettings())
    with pytest.raises(ValueError, match="finite"):
        blsmod._grid_segments(cb.GridSpec(kind="frequency", values=np.linspace(0.0, 0.5, 20)),
                              cb.BLSSettings())


def _method_cases():
    index = json.load(open(os.path.join(GOLDEN, "method_cases.json")))
    z = np.load(os.path.join(GOLDEN, "method_cases.npz"))
    return [(m, z) for m in index]


@pytest.mark.parametrize("case", _method_cases(), ids=lambda c: c[0]["name"])
def test_peaks_and_row_match_reference(case):
    """The reference's spectrum through this package's Periodogram: same best
    period, same alias-diverse peak list and same batch row."""
    meta, z = case
    k = meta["key"]
    extras = {name: z[f"{k}_x_{name}"] for name in ("depth", "depth_snr", "duration", "t0", "sde")}
    pg = Periodogram.from_spectrum(method="BLS", backend="numba", frequency=z[f"{k}_frequency"],
                                   power=z[f"{k}_power"], objective_sense="max",
                                   n_samples=meta["n_samples"], baseline=meta["baseline"],
                                   extras=extras).with_peak_defaults(cb.BLSSettings(**meta["settings"]))
    assert pg.best_period() == meta["best_period"]
    peaks = [p.to_dict() for p in pg.best_periods(10, alias_diverse=True)]
    assert peaks == meta["peaks"]
    row = periodogram_to_row(meta["name"], pg, n_best=10, alias_diverse=True)
    ref = {k2: (float("nan") if v is None else v) for k2, v in meta["row"].items()}
    assert set(row) == set(ref)
    for key, v in ref.items():
        if isinstance(v, float) and np.isnan(v):
            assert np.isnan(row[key]), key
        else:
            assert row[key] == v, key


def test_segment_grids_of_method_cases_match_reference():
    for meta, z in _method_cases():
        s = cb.BLSSettings(**meta["settings"])
        grid = cb.GridSpec(kind="period", values=z[f"{meta['key']}_grid"],
                           meta=meta["grid_meta"] if meta["grid_meta"] else {})
        segs = blsmod._grid_segments(grid, s)
        assert sum(p.size for p, _ in segs) == grid.size


def test_argument_errors_raise_before_any_device_work():
    t = np.linspace(0.0, 10.0, 100)
    with pytest.raises(ValueError, match="objective"):
        cb.bls_power(t, np.ones(100), np.ones(100), np.array([1.0]), np.array([0.1]), 10,
                     objective="chi2")
    with pytest.raises(ValueError, match="backend"):
        cb.bls_power(t, np.ones(100), np.ones(100), np.array([1.0]), np.array([0.1]), 10,
                     backend="numba")
    out = cb.bls_power(t, np.ones(100), np.ones(100), np.zeros(0), np.array([0.1]), 10)
    assert out.power.size == 0
    with pytest.raises(cb.BackendUnavailableError):
        cb.BLSMethod().resolve_backend("astropy")
    with pytest.raises(cb.UnknownMethodError):
        cb.get_method("GLS")

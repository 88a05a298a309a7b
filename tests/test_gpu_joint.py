"""The joint-ephemeris ("shared") multi-band search on the engine: against the
reference's golden output (tests/golden/make_golden_multiband.py, the numba
joint sweep) and against the oracle's restatement of that sweep on seeded
stars, including the histograms-in-global-memory path and stars where no box
is admissible.

The engine's box sums are exact 64-bit fixed-point sums; the reference's are
sequential FP64 sums.  Values therefore agree to rounding (relative 1e-6 is
asserted) and the chosen box agrees except where two boxes tie to rounding."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from test_multiband_host import _cases, mblc_of

pytestmark = pytest.mark.gpu

FIELDS = ("power", "depth", "depth_snr", "duration", "transit_time", "band_index")


@pytest.mark.parametrize("case", [c for c in _cases() if c[0]["ephemeris"] == "shared"],
                         ids=lambda c: c[0]["key"])
def test_shared_matches_reference(case):
    from cuperiod_b200.api import periodogram
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    meta, z = case
    k = meta["key"]
    settings = BLSSettings(objective=meta["objective"], mb_ephemeris="shared")
    grid = GridSpec(kind="period", values=z[f"{k}_periods"]) if meta["explicit_grid"] else None
    pg = periodogram(mblc_of(meta, z), "BLS", grid=grid, settings=settings)
    assert pg.meta["mb_ephemeris"] == "shared"
    assert list(pg.meta["bands"]) == meta["used_bands"]
    assert pg.n_samples == meta["n_samples"] and pg.baseline == meta["baseline"]
    np.testing.assert_array_equal(pg.frequency, z[f"{k}_frequency"])
    ref = z[f"{k}_power"]
    same = ((pg.extras["duration"] == z[f"{k}_x_duration"])
            & (np.abs(pg.extras["t0"] - z[f"{k}_x_t0"]) <= 1e-9)
            & (pg.extras["band_index"] == z[f"{k}_x_band_index"]))
    assert same.mean() >= 0.99
    np.testing.assert_allclose(pg.power[same], ref[same], rtol=1e-6, atol=1e-9 * float(ref.max()))
    np.testing.assert_allclose(pg.extras["depth"][same], z[f"{k}_x_depth"][same], rtol=1e-6,
                               atol=1e-12)
    if meta["objective"] == "snr":
        # the box maximises the summed squared SNRs, which is the power: a box
        # chosen differently on a near tie still has (nearly) the same power
        np.testing.assert_allclose(pg.power, ref, rtol=1e-6, atol=1e-9 * float(ref.max()))
        np.testing.assert_allclose(pg.extras["sde"], z[f"{k}_x_sde"], rtol=1e-5, atol=1e-6)
    assert pg.best_period() == meta["best_period"]


def _star(rng, n_bands, *, n=(200, 900), span=30.0, period=2.2, depth=3e-3, same_time=False):
    bands = []
    for b in range(n_bands):
        m = int(rng.integers(*n))
        t = (np.full(m, 5.0) if same_time
             else np.sort(rng.uniform(0.0, span, m)) + 2459000.0 + rng.uniform(0, 5))
        level = float(rng.uniform(0.5, 4.0))
        noise = float(rng.uniform(1e-3, 5e-3))
        y = level * (1.0 + rng.normal(0.0, noise, m))
        y[np.mod(t - 0.3, period) < 0.07] -= level * depth * rng.uniform(0.5, 1.5)
        dy = level * noise * rng.uniform(0.7, 1.3, m)
        bands.append((t, y, dy))
    return bands


def _engine_vs_oracle(bands, periods, durations_per_seg, oversample, objective):
    from cuperiod_b200 import _lib
    segs = list(zip(periods, durations_per_seg))
    grid = _lib.PackedGrid.from_segments(segs, oversample, objective)
    packed = _lib.PackedCurves.from_arrays(bands)
    got = _lib.default_engine().search_joint(grid, packed)
    jb = oracle.joint_bands([b[0] for b in bands], [b[1] for b in bands], [b[2] for b in bands])
    ref = {f: [] for f in FIELDS}
    for per, dur in segs:
        o = oracle.joint_power(jb, per, dur, oversample, objective, n_threads=8)
        for f in FIELDS:
            ref[f].append(o[f])
    return dict(zip(FIELDS, got)), {f: np.concatenate(v) for f, v in ref.items()}


def _agree(got, ref, min_same=0.99):
    same = ((got["duration"] == ref["duration"])
            & (np.abs(got["transit_time"] - ref["transit_time"]) <= 1e-9)
            & (got["band_index"] == ref["band_index"]))
    assert same.mean() >= min_same
    for f in ("power", "depth", "depth_snr"):
        np.testing.assert_allclose(got[f][same], ref[f][same], rtol=1e-6,
                                   atol=1e-9 * max(float(np.abs(ref[f]).max()), 1e-300))
    return same


@pytest.mark.parametrize("objective", [0, 1])
@pytest.mark.parametrize("n_bands", [1, 4])
def test_joint_matches_oracle(n_bands, objective):
    rng = np.random.default_rng(100 + 10 * n_bands + objective)
    bands = _star(rng, n_bands)
    seg_p = [np.geomspace(0.6, 1.2, 900), np.geomspace(1.2, 2.4, 900), np.geomspace(2.4, 4.8, 900)]
    seg_d = [np.geomspace(0.012, 0.15, 8) * p[0] / 0.6 for p in seg_p]
    got, ref = _engine_vs_oracle(bands, seg_p, seg_d, 10, objective)
    _agree(got, ref)


def test_joint_many_bands_global_histograms():
    # 40 bands x 2 histograms x ~2000 bins exceed one CTA's shared memory: the
    # kernel keeps them in a global slice per CTA
    rng = np.random.default_rng(7)
    bands = _star(rng, 40, n=(20, 60))
    seg_p = [np.geomspace(4.0, 8.0, 300)]
    seg_d = [np.geomspace(0.04, 0.48, 8)]
    got, ref = _engine_vs_oracle(bands, seg_p, seg_d, 10, 0)
    _agree(got, ref)


def test_joint_no_admissible_box():
    # every point at one time: each box holds all or none of a band's weight,
    # so no box is admissible and every field is 0, as in the reference
    rng = np.random.default_rng(3)
    bands = _star(rng, 3, n=(5, 9), same_time=True)
    seg_p = [np.geomspace(1.0, 2.0, 50)]
    seg_d = [np.array([0.05, 0.1, 0.2])]
    got, ref = _engine_vs_oracle(bands, seg_p, seg_d, 10, 0)
    for f in FIELDS:
        assert np.all(ref[f] == 0.0)
        np.testing.assert_array_equal(got[f], ref[f])


def test_joint_rejects_bad_input():
    from cuperiod_b200 import _lib
    grid = _lib.PackedGrid.from_segments([(np.array([1.0, 2.0]), np.array([0.1]))], 10, 0)
    bad = _lib.PackedCurves.from_arrays([(np.array([0.0, 1.0, np.nan]), np.ones(3), None)])
    with pytest.raises(ValueError, match="finite"):
        _lib.default_engine().search_joint(grid, bad)

"""The TLS matched filter on the engine against the reference's golden output
(tests/golden/make_golden_tls.py, the numba kernel) and the oracle's restatement
of that kernel on seeded curves.

The engine's phase bins are the reference's bit for bit; its bin sums are exact
sums of 64-bit fixed-point values rounded once to FP64 where the reference adds
FP64 values in point order, and from the bins on every operation is the
reference's.  Values
agree to rounding and the winning template and start agree except on near
ties."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from test_oracle_tls import case_inputs, tls_cases

pytestmark = pytest.mark.gpu


def _agree(got, ref, min_same=0.99, rtol=1e-7):
    same = (got["duration"] == ref["duration"]) & (np.abs(got["t0"] - ref["t0"]) <= 1e-9)
    assert same.mean() >= min_same, same.mean()
    np.testing.assert_allclose(got["sr"][same], ref["sr"][same], rtol=rtol,
                               atol=1e-12 * max(float(np.max(np.abs(ref["sr"]))), 1e-300))
    np.testing.assert_allclose(got["depth"][same], ref["depth"][same], rtol=rtol,
                               atol=1e-12 * max(float(np.max(np.abs(ref["depth"]))), 1e-300))
    np.testing.assert_allclose(got["sde"], ref["sde"], rtol=1e-6, atol=1e-6)
    assert int(np.argmax(got["sde"])) == int(np.argmax(ref["sde"]))
    return same


@pytest.mark.parametrize("case", tls_cases(), ids=lambda c: c[0]["key"])
def test_tls_matches_reference(case):
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import tls_power
    meta, z = case
    t, y, dy, periods, _ = case_inputs(meta, z)
    got = tls_power(t, y, dy, periods, settings=TLSSettings(**meta["settings"]))
    ref = {k: z[f"{meta['key']}_{k}"] for k in meta["outputs"]}
    if meta["key"] == "constant_flux":
        for k in ref:
            np.testing.assert_array_equal(got[k], ref[k])
        return
    _agree(got, ref)


def _curve(seed, n, *, span=30.0, period=2.3, depth=3e-3, noise=1e-3, with_error=True):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0.0, span, n)) + 1500.0
    y = 1.0 + rng.normal(0.0, noise, n)
    ph = np.mod(t - 0.7, period) / period
    y[np.minimum(ph, 1.0 - ph) < 0.015] -= depth
    dy = noise * rng.uniform(0.6, 1.4, n) if with_error else None
    return t, y, dy


@pytest.mark.parametrize("n,n_bins,with_error", [(37, 256, True), (2048, 256, False),
                                                 (5000, 300, True), (9000, 1024, True)])
def test_tls_matches_oracle(n, n_bins, with_error):
    # short curves (tail only), exactly one chunk, chunks plus a tail; several
    # bin counts (and so template widths and tiles per work item)
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import tls_power
    t, y, dy = _curve(n, n, with_error=with_error)
    s = TLSSettings(n_phase_bins=n_bins)
    periods = np.geomspace(0.6, 12.0, 1500)
    got = tls_power(t, y, dy, periods, settings=s)
    ref = oracle.tls_power(t, y, dy, periods, n_bins=n_bins, n_threads=8)
    _agree(got, ref)


def test_tls_batch_equals_single_curves():
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import tls_power, tls_power_many
    curves = [_curve(10 + i, 400 + 700 * i, with_error=i % 2 == 0) for i in range(5)]
    curves.append((curves[0][0], np.full(curves[0][0].size, 2.0), None))   # constant
    periods = np.geomspace(0.7, 9.0, 800)
    s = TLSSettings()
    many = tls_power_many(curves, periods, settings=s)
    for c, got in zip(curves, many):
        one = tls_power(*c, periods, settings=s)
        for k in one:
            np.testing.assert_array_equal(got[k], one[k])


def test_tls_periodogram_recovers_the_transit():
    from cuperiod_b200.api import periodogram
    t, y, dy = _curve(77, 4000, span=40.0, period=3.1, depth=2e-3)
    pg = periodogram((t, y, dy), "TLS", domain="flux")
    assert abs(pg.best_period() - 3.1) / 3.1 < 3e-3
    assert pg.method == "TLS" and list(pg.extras)[:4] == ["sr", "depth", "duration", "t0"]


def test_tls_rejects_bad_input():
    from cuperiod_b200 import _lib
    eng = _lib.default_engine()
    tau = np.linspace(0.0, 10.0, 50)
    good = dict(n_bins=64, dur_bins=[2, 4], templates={2: np.ones(2), 4: np.ones(4)},
                den_rel=1e-9)
    with pytest.raises(ValueError, match="finite"):
        eng.tls_search([(tau, np.full(50, np.nan), np.ones(50), 50.0)], [1.0, 2.0], **good)
    with pytest.raises(ValueError, match="template width"):
        eng.tls_search([(tau, np.zeros(50), np.ones(50), 50.0)], [1.0],
                       **{**good, "dur_bins": [64], "templates": {64: np.ones(64)}})
    with pytest.raises(ValueError, match="periods"):
        eng.tls_search([(tau, np.zeros(50), np.ones(50), 50.0)], [0.0], **good)


def test_tls_long_curve_bins_stay_exact():
    # 600,000 points, many per bin: the fold's carry-propagating 32-bit atomics
    # keep every bin's int64 sum exact at any count
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import tls_power
    t, y, dy = _curve(5, 600_000, span=400.0, period=4.7, depth=5e-4, noise=2e-3)
    periods = np.array([1.3, 4.7, 9.1])
    got = tls_power(t, y, dy, periods, settings=TLSSettings())
    ref = oracle.tls_power(t, y, dy, periods, n_threads=8)
    np.testing.assert_array_equal(got["duration"], ref["duration"])
    np.testing.assert_array_equal(got["t0"], ref["t0"])
    np.testing.assert_allclose(got["sr"], ref["sr"], rtol=1e-9)


def test_tls_batch_rows():
    # batch_periodograms with method="TLS": one launch per chunk of curves that
    # share a grid, rows with the reference's TLS peak columns; a short curve is
    # recorded as an error, as the reference's runner records it
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import TLSSettings
    curves = [_curve(30 + i, 1500) for i in range(3)]
    grid = GridSpec(kind="period", values=np.geomspace(0.7, 9.0, 600))
    t0, y0, _ = curves[0]
    inputs = [(f"c{i}", c) for i, c in enumerate(curves)] + [("short", (t0[:5], y0[:5]))]
    out = batch_periodograms(inputs, "TLS", grid=grid, settings=TLSSettings(), domain="flux",
                             n_best=3)
    assert [r["key"] for r in out.rows] == ["c0", "c1", "c2"] and "short" in out.errors
    row = out.rows[0]
    assert row["method"] == "TLS" and {"sr_1", "depth_1", "duration_1", "t0_1"} <= set(row)
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.tls import TLSMethod
    pg = TLSMethod().power(grid, LightCurve(*curves[0], Domain.FLUX), TLSSettings())
    assert row["best_period"] == pg.best_period()

"""Batch result rows with the peaks ranked on the device against the reference's
row of the host-assembled periodogram (periodogram_to_row, alias-diverse)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from tests._cases import transit_curve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from cuperiod_b200 import _lib
    eng = _lib.Engine()
    yield eng
    eng.close()


def _keyed():
    from cuperiod_b200.lightcurve import Domain, LightCurve
    specs = [(900, 2.3, 4e-3, 11, "uniform"), (2500, 4.1, 3e-3, 12, "hetero"),
             (1700, 1.7, 5e-3, 13, "uniform"), (600, 6.2, 6e-3, 14, "wild"),
             (3000, 3.3, 2e-3, 15, "uniform"), (1200, 3.0, 0.0, 16, "uniform")]
    out = []
    for i, (n, p, depth, seed, w) in enumerate(specs):
        t, y, dy = transit_curve(n, span=27.0, period=p, depth=depth, seed=seed, weights=w)
        out.append((f"c{i}", LightCurve(t, y, dy, domain=Domain.FLUX)))
    return out


def _host_rows(keyed, grid_of, settings, engine, n_best):
    from cuperiod_b200.batch import PEAK_EXTRA_COLUMNS, periodogram_to_row
    from cuperiod_b200.bls import BLSMethod
    m = BLSMethod()
    rows = []
    for key, lc in keyed:
        pg = m.power_many(grid_of(lc), [lc], settings, engine=engine)[0]
        rows.append(periodogram_to_row(key, pg.with_peak_defaults(settings), n_best=n_best,
                                       extra_keys=PEAK_EXTRA_COLUMNS, alias_diverse=True))
    return rows


def _same_row(dev, host):
    assert list(dev) == list(host)
    for k, b in host.items():
        a = dev[k]
        if isinstance(b, float):
            if k.startswith("sde_"):            # mean and std summed in another order
                assert (math.isnan(a) and math.isnan(b)) or abs(a - b) <= 1e-9 * max(1.0, abs(b)), k
            else:
                assert a == b or (math.isnan(a) and math.isnan(b)), (k, a, b)
        else:
            assert a == b, (k, a, b)


def _rows_of_same_launch(engine, grid, keyed, s, n_best):
    """Device rows, and host rows of the same launch's spectra (per-point-weight
    sums are FP64 in atomic order, so two launches may differ in the last bits)."""
    from cuperiod_b200.batch import PEAK_EXTRA_COLUMNS, periodogram_to_row
    from cuperiod_b200.bls import BLSMethod, _assemble, _fields, _grid_segments, _prepared_curve
    dev = BLSMethod().rows_many(grid, keyed, s, n_best=n_best, extra_keys=PEAK_EXTRA_COLUMNS,
                                engine=engine)
    out = engine.download()
    segments = _grid_segments(grid, s)
    host = []
    for i, (key, lc) in enumerate(keyed):
        f, _ = _prepared_curve(lc, s)
        pg = _assemble(_fields(out[:, i, :], segments), f.n, f.baseline, f.meta)
        host.append(periodogram_to_row(key, pg.with_peak_defaults(s), n_best=n_best,
                                       extra_keys=PEAK_EXTRA_COLUMNS, alias_diverse=True))
    return dev, host


def test_device_rows_equal_host_rows(engine):
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    grid = GridSpec(kind="period", values=np.geomspace(0.5, 12.0, 20000))
    dev, host = _rows_of_same_launch(engine, grid, _keyed(), s, 10)
    for d, h in zip(dev, host):
        _same_row(d, h)
    assert all(not math.isnan(d["period_10"]) for d in dev[:5])


def test_batch_rows_on_default_grids(engine):
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    # one weight per curve: exact integer sums, identical in any launch
    keyed = [kv for kv in _keyed() if np.all(kv[1].error == kv[1].error[0])]
    summary = batch_periodograms(keyed, grid=None, settings=s, n_best=10, engine=engine)
    assert not summary.errors
    host = _host_rows(keyed, lambda lc: BLSMethod().default_grid(lc, s), s, engine, 10)
    by_key = {r["key"]: r for r in summary.rows}
    for h in host:
        _same_row(by_key[h["key"]], h)


@pytest.mark.parametrize("n_periods", [1, 2, 3])
def test_device_rows_on_tiny_grids(engine, n_periods):
    from cuperiod_b200.batch import PEAK_EXTRA_COLUMNS
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    grid = GridSpec(kind="period", values=np.array([2.1, 2.7, 3.3][:n_periods]))
    dev, host = _rows_of_same_launch(engine, grid, _keyed()[:3], s, 3)
    for d, h in zip(dev, host):
        _same_row(d, h)


def test_threaded_batch_rows_equal_single_threaded():
    # curves with distinct baselines get distinct default grids; chunks of 5
    # curves (each chunk one launch over its curves' own grids) run on worker
    # threads with their own engines and must give the rows of a
    # single-threaded run, in order
    import numpy as np

    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.synthetic import batched_curves
    rng = np.random.default_rng(8)
    inputs = []
    for i, c in enumerate(batched_curves(24, seed=9, n_range=(500, 3000))):
        keep = c.t < c.t.min() + rng.uniform(15.0, 27.0)
        inputs.append((f"c{i}", (c.t[keep], c.y[keep])))
    one = batch_periodograms(inputs, "BLS", domain="flux", workers=1, n_best=3, chunk_size=5)
    many = batch_periodograms(inputs, "BLS", domain="flux", workers=4, n_best=3, chunk_size=5)
    assert one.launches == many.launches == 5
    assert [r["key"] for r in many.rows] == [f"c{i}" for i in range(24)]
    assert many.rows == one.rows
    # and one launch for the whole catalogue gives the same rows
    whole = batch_periodograms(inputs, "BLS", domain="flux", n_best=3)
    assert whole.launches == 1 and whole.rows == one.rows


def test_threaded_batch_of_stars_and_curves_equals_single_threaded():
    # multi-band stars are launches of their own beside the single-band chunks;
    # threaded and single-threaded runs give the same rows in the same order
    # and record the same failures
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.lightcurve import Domain, LightCurve, MultiBandLightCurve
    from cuperiod_b200.settings import BLSSettings
    from cuperiod_b200.synthetic import batched_curves, multiband_stars
    inputs = []
    for i, star in enumerate(multiband_stars(3, seed=21, n_range=(600, 1200))):
        inputs.append((f"s{i}", MultiBandLightCurve.from_light_curves(
            {b: LightCurve(c.t, c.y, c.dy, Domain.FLUX) for b, c in star.items()})))
    for i, c in enumerate(batched_curves(4, seed=22, n_range=(500, 1500))):
        inputs.append((f"c{i}", (c.t, c.y)))
    inputs.append(("short", MultiBandLightCurve.from_light_curves({
        "g": LightCurve(np.arange(2.0), np.ones(2), None, Domain.FLUX)})))
    s = BLSSettings(mb_ephemeris="shared")
    one = batch_periodograms(inputs, "BLS", domain="flux", settings=s, workers=1, n_best=3)
    many = batch_periodograms(inputs, "BLS", domain="flux", settings=s, workers=4, n_best=3)
    assert [r["key"] for r in many.rows][:3] == ["s0", "s1", "s2"]
    assert len(many.rows) == 7 and many.launches == one.launches
    assert many.errors == one.errors and list(many.errors) == ["short"]
    assert many.rows == one.rows


def test_concurrent_launches_with_different_shared_memory_needs():
    # a launch raises its kernel's dynamic shared-memory limit, which is one
    # value per kernel and device for the whole process: threads whose batches
    # need different amounts (the peak ranking's candidate mask grows with the
    # grid) must never lower it under one another
    from concurrent.futures import ThreadPoolExecutor

    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    keyed = _keyed()[:2]
    sizes = [60000, 2000, 45000, 3000, 30000, 5000, 20000, 1000] * 3

    def job(n_periods):
        grid = GridSpec(kind="period", values=np.geomspace(0.5, 12.0, n_periods))
        return BLSMethod().rows_many(grid, keyed, s, n_best=3, engine=_lib.default_engine())

    with ThreadPoolExecutor(max_workers=4) as pool:
        results = list(pool.map(job, sizes))
    assert all(len(r) == 2 and r[0]["key"] == keyed[0][0] for r in results)
    # the same grid gives the same rows whichever thread ran it
    for n in set(sizes):
        runs = [r for r, k in zip(results, sizes) if k == n]
        assert all(run == runs[0] for run in runs)

"""One launch over curves with their own trial grids (bls_prepare_grids)
against one launch per grid: the same spectra, bests and result rows."""

from __future__ import annotations

import numpy as np
import pytest

from _cases import transit_curve

pytestmark = pytest.mark.gpu


def _grids_and_curves(objective: int):
    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import BLSMethod, _grid_segments
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings(objective="likelihood" if objective else "snr")
    m = BLSMethod()
    specs = [(1400, 9.0, "uniform", 1), (900, 14.0, "uniform", 2), (2600, 20.0, "hetero", 3),
             (700, 9.0, "wild", 4), (1800, 27.0, "uniform", 5), (1100, 14.0, "hetero", 6),
             (500, 20.0, "uniform", 7)]
    curves, grids = [], {}
    for n, span, w, seed in specs:
        t, y, dy = transit_curve(n, span=span, weights=w, seed=seed, period=2.1)
        lc = LightCurve(t, y, dy, Domain.FLUX)
        if span not in grids:
            grids[span] = m.default_grid(lc, s)      # the default grid of this baseline
        curves.append((t, y, dy, span))
    # an explicit grid of its own beside the default ones
    grids["explicit"] = GridSpec(kind="period", values=np.geomspace(0.4, 5.0, 2500))
    t, y, dy = transit_curve(1300, span=12.0, seed=8, period=1.3)
    curves.insert(3, (t, y, dy, "explicit"))
    names = list(grids)
    packed = [_lib.PackedGrid.from_segments(_grid_segments(grids[k], s), s.bins_per_duration,
                                            objective) for k in names]
    gid = [names.index(c[3]) for c in curves]
    return packed, gid, curves


@pytest.mark.parametrize("objective", [0, 1])
def test_one_launch_over_many_grids_equals_a_launch_per_grid(objective):
    from cuperiod_b200 import _lib
    grids, gid, curves = _grids_and_curves(objective)
    eng = _lib.Engine()
    try:
        eng.prepare_grids(grids, gid, _lib.PackedCurves.from_arrays(
            [(t, y, dy) for t, y, dy, _ in curves]))
        info = eng.info()
        eng.launch()
        flat = eng.download_flat()
        off = eng.spectrum_offsets
        best = eng.download_best()
        alone = []
        for (t, y, dy, _), k in zip(curves, gid):
            alone.append(eng.search(grids[k], _lib.PackedCurves.from_arrays([(t, y, dy)]))[:, 0])
    finally:
        eng.close()
    assert info["n_grids"] == len(grids)
    assert info["spectrum"] == sum(grids[k].n_periods for k in gid) == off[-1]
    for c, ref in enumerate(alone):
        got = flat[:, off[c]:off[c + 1]]
        assert got.shape == ref.shape
        dy = curves[c][2]
        if dy is not None and (dy.max() / dy.min()) ** 2 > 256.0:
            # FP64 sums in atomic order: equal to rounding, same best
            fin = np.isfinite(ref[0])
            np.testing.assert_array_equal(np.isfinite(got[0]), fin)
            np.testing.assert_allclose(got[0][fin], ref[0][fin], rtol=1e-9)
        else:
            np.testing.assert_array_equal(got, ref)
        p = np.nan_to_num(got[0], nan=0.0, posinf=0.0, neginf=0.0)
        assert best[0][c] == int(np.argmax(p))
        np.testing.assert_allclose(best[2][c], p.mean(), rtol=1e-12)


def test_rows_by_grid_equal_rows_of_each_grid():
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import BLSSettings
    s = BLSSettings()
    m = BLSMethod()
    items = []
    for i, (n, span, seed) in enumerate([(1200, 10.0, 21), (800, 16.0, 22), (2000, 23.0, 23),
                                         (1500, 10.0, 24), (600, 16.0, 25)]):
        t, y, dy = transit_curve(n, span=span, seed=seed, period=1.9)
        lc = LightCurve(t, y, dy, Domain.FLUX)
        items.append((f"k{i}", lc))
    grids = {}
    for key, lc in items:
        grids.setdefault(lc.baseline // 1.0, m.default_grid(lc, s))
    triples = [(key, lc, grids[lc.baseline // 1.0]) for key, lc in items]
    together = m.rows_by_grid(triples, s, n_best=4)
    each = [m.rows_many(g, [(key, lc)], s, n_best=4)[0] for key, lc, g in triples]
    assert [r["key"] for r in together] == [f"k{i}" for i in range(5)]
    assert together == each


def _same_rows(a, b, loose=()):
    """Rows equal field by field (NaN equal to NaN); for the keys in ``loose``
    (FP64 sums in atomic order) floats within 1e-9 relative."""
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.keys() == y.keys()
        for k in x:
            vx, vy = x[k], y[k]
            if isinstance(vx, float) and isinstance(vy, float):
                if vx != vx and vy != vy:
                    continue
                if x["key"] in loose:
                    assert abs(vx - vy) <= 1e-9 * max(abs(vx), abs(vy)), (x["key"], k, vx, vy)
                    continue
            assert vx == vy, (x["key"], k, vx, vy)


def test_native_default_grids_give_the_rows_of_python_default_grids():
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import BLSSettings
    m = BLSMethod()
    keyed = []
    for i, (n, span, w, seed) in enumerate([(900, 8.5, "uniform", 31), (1500, 13.2, "hetero", 32),
                                            (2400, 27.0, "uniform", 33), (700, 8.5, "wild", 34),
                                            (400, 5.1, "uniform", 35), (3000, 44.0, "hetero", 36)]):
        t, y, dy = transit_curve(n, span=span, weights=w, seed=seed, period=1.7)
        keyed.append((f"d{i}", LightCurve(t, y, dy, Domain.FLUX)))
    for s in (BLSSettings(), BLSSettings(objective="likelihood", grid_oversample=3)):
        native = m.rows_default(keyed, s, n_best=12)
        python = m.rows_by_grid([(k, lc, m.default_grid(lc, s)) for k, lc in keyed], s,
                                n_best=12)
        _same_rows(native, python, loose=("d3",))   # d3: weights over four decades
    # the batch runner takes the native path and records the same failures
    short = ("short", LightCurve(np.linspace(0.0, 0.3, 40), np.ones(40), None, Domain.FLUX))
    res = batch_periodograms(keyed + [short], "BLS", n_best=12)
    assert res.launches == 1 and list(res.errors) == ["short"]
    from cuperiod_b200.batch import PEAK_EXTRA_COLUMNS
    _same_rows(res.rows, m.rows_default(keyed, BLSSettings(), n_best=12,
                                        extra_keys=PEAK_EXTRA_COLUMNS), loose=("d3",))

"""Method-level parity on the GPU: ``periodogram(lc, "BLS")``,
``BLSMethod().power`` and the batch row through the engine against the
reference's own outputs for the same curves (``tests/golden/method_cases.*``,
made by ``BLSMethod.power(grid, lc, settings, "numba")`` and
``periodogram_to_row``, src/cuperiod/methods/bls.py:361-395 and
src/cuperiod/batch/io.py:507-571).

Tolerances: frequencies and the best period are equal; power within 1e-6
relative (floor 1e-9 of the largest power); where the engine picked the
reference's box (same duration and mid-transit time) depth and depth_snr within
1e-6 relative; SDE within 1e-6 absolute; the row's peak periods equal and its
powers within 1e-6 relative.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from _cases import GOLDEN

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def _cases():
    index = json.load(open(os.path.join(GOLDEN, "method_cases.json")))
    z = np.load(os.path.join(GOLDEN, "method_cases.npz"))
    return [(m, z) for m in index]


def _inputs(meta, z):
    import cuperiod_b200 as cb
    k = meta["key"]
    lc = cb.LightCurve.from_arrays(z[f"{k}_t"], z[f"{k}_flux"], z[f"{k}_err"],
                                   domain=cb.Domain.FLUX)
    settings = cb.BLSSettings(**meta["settings"])
    grid = None
    if not meta["grid_meta"]:
        grid = cb.GridSpec(kind="period", values=z[f"{k}_grid"])
    return lc, settings, grid


def _check_spectrum(pg, meta, z):
    k = meta["key"]
    np.testing.assert_array_equal(pg.frequency, z[f"{k}_frequency"])
    ref = z[f"{k}_power"]
    scale = float(np.max(np.abs(ref)))
    err = np.abs(pg.power - ref)
    assert np.all(err <= RTOL * np.abs(ref) + 1e-9 * scale), float(err.max())
    same = (pg.extras["duration"] == z[f"{k}_x_duration"]) & (
        np.abs(pg.extras["t0"] - z[f"{k}_x_t0"]) <= 1e-9)
    assert same.mean() >= 0.99, same.mean()
    for name in ("depth", "depth_snr"):
        r, g = z[f"{k}_x_{name}"][same], pg.extras[name][same]
        assert np.all(np.abs(g - r) <= RTOL * np.abs(r) + 1e-12 * np.abs(r).max()), name
    np.testing.assert_allclose(pg.extras["sde"], z[f"{k}_x_sde"], rtol=0.0, atol=1e-6)
    assert pg.best_period() == meta["best_period"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0]["name"])
def test_periodogram_matches_the_reference(case):
    import cuperiod_b200 as cb
    meta, z = case
    lc, settings, grid = _inputs(meta, z)
    pg = cb.periodogram(lc, "BLS", settings=settings, grid=grid)
    _check_spectrum(pg, meta, z)
    peaks = [p.to_dict() for p in pg.best_periods(10, alias_diverse=True)]
    assert [p["period"] for p in peaks] == [p["period"] for p in meta["peaks"]]
    for p, r in zip(peaks, meta["peaks"]):
        assert abs(p["power"] - r["power"]) <= RTOL * abs(r["power"])


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0]["name"])
def test_method_power_and_batch_row_match_the_reference(case):
    import cuperiod_b200 as cb
    meta, z = case
    lc, settings, grid = _inputs(meta, z)
    m = cb.BLSMethod()
    g = grid or m.default_grid(lc, settings)
    np.testing.assert_array_equal(np.sort(g.period), np.sort(z[f"{meta['key']}_grid"]))
    _check_spectrum(m.power(g, lc, settings).with_peak_defaults(settings), meta, z)
    # the batch entry: the row's peaks ranked on the device
    summary = cb.batch_periodograms([(meta["name"], lc)], "BLS", grid=grid, settings=settings,
                                    n_best=10)
    assert not summary.errors and len(summary.rows) == 1
    row, ref = summary.rows[0], meta["row"]
    assert row["best_period"] == ref["best_period"]
    for j in range(1, 11):
        rp, gp = ref.get(f"period_{j}"), row.get(f"period_{j}")
        if rp is None:
            assert gp is None or np.isnan(gp)
            continue
        assert gp == rp, j
        assert abs(row[f"power_{j}"] - ref[f"power_{j}"]) <= RTOL * abs(ref[f"power_{j}"])

"""Multi-band host logic against the reference's golden output: the stacked
default grid, band selection and the error rule (no GPU needed)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from _cases import GOLDEN


def _cases():
    index = json.load(open(os.path.join(GOLDEN, "multiband_cases.json")))
    z = np.load(os.path.join(GOLDEN, "multiband_cases.npz"))
    return [(m, z) for m in index]


def mblc_of(meta, z):
    from cuperiod_b200.lightcurve import Domain, LightCurve, MultiBandLightCurve
    k = meta["key"]
    return MultiBandLightCurve.from_light_curves({
        b: LightCurve(z[f"{k}_{b}_t"], z[f"{k}_{b}_y"], z[f"{k}_{b}_dy"] if has else None,
                      Domain.FLUX)
        for b, has in zip(meta["bands"], meta["with_error"])})


@pytest.mark.parametrize("case", [c for c in _cases() if not c[0]["explicit_grid"]],
                         ids=lambda c: c[0]["key"])
def test_default_grid_over_stacked_baseline(case):
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.multiband import multiband_default_grid
    from cuperiod_b200.settings import BLSSettings
    meta, z = case
    g = multiband_default_grid(BLSMethod(), mblc_of(meta, z), BLSSettings())
    np.testing.assert_array_equal(g.period, z[f"{meta['key']}_periods"])
    for k, v in meta["grid_meta"].items():
        got = g.meta[k]
        assert (list(got) if isinstance(got, tuple) else got) == v


def test_band_rules():
    from cuperiod_b200.lightcurve import Domain, LightCurve, MultiBandLightCurve
    from cuperiod_b200.multiband import band_errors, resolve_ephemeris, robust_scatter
    rng = np.random.default_rng(0)
    a = LightCurve(np.arange(50.0), 1 + rng.normal(0, 1e-3, 50), np.full(50, 2e-3), Domain.FLUX)
    b = LightCurve(np.arange(40.0), 2 + rng.normal(0, 3e-3, 40), None, Domain.FLUX)
    errs = band_errors([a, b])                        # one band lacks errors: both scatter
    assert errs[0][0] == robust_scatter(a.value) and errs[1][0] == robust_scatter(b.value)
    assert band_errors([a, a])[0] is not None and np.array_equal(band_errors([a, a])[0], a.error)
    assert robust_scatter(np.ones(10)) == 1.0
    assert resolve_ephemeris(None) == "independent"
    with pytest.raises(ValueError):
        resolve_ephemeris(None, "joint")
    with pytest.raises(ValueError):
        MultiBandLightCurve({"g": a, "m": LightCurve(np.arange(3.0), np.ones(3))})


@pytest.mark.parametrize("ephemeris", ["independent", "shared"])
def test_band_selection_fails_before_the_device(ephemeris):
    from cuperiod_b200.errors import InsufficientDataError
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.lightcurve import Domain, LightCurve, MultiBandLightCurve
    from cuperiod_b200.multiband import bls_multiband_power
    from cuperiod_b200.settings import BLSSettings
    short = MultiBandLightCurve.from_light_curves({
        "g": LightCurve(np.arange(2.0), np.ones(2), None, Domain.FLUX),
        "r": LightCurve(np.arange(2.0) + 0.5, np.ones(2), None, Domain.FLUX)})
    with pytest.raises(InsufficientDataError, match="no band has enough"):
        bls_multiband_power(GridSpec(kind="period", values=np.array([1.0, 2.0])), short,
                            BLSSettings(), ephemeris=ephemeris)


def test_batch_records_short_stars_and_curves_without_a_launch():
    # a star whose bands are all too short fails when its launch would start,
    # in a worker; like a short single-band curve it lands in ``errors`` and no
    # engine is created (there is nothing to launch)
    from cuperiod_b200.batch import batch_periodograms
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.lightcurve import Domain, LightCurve, MultiBandLightCurve
    short = MultiBandLightCurve.from_light_curves({
        "g": LightCurve(np.arange(2.0), np.ones(2), None, Domain.FLUX),
        "r": LightCurve(np.arange(2.0) + 0.5, np.ones(2), None, Domain.FLUX)})
    grid = GridSpec(kind="period", values=np.array([1.0, 2.0]))
    res = batch_periodograms([("star", short), ("curve", (np.arange(3.0), np.ones(3)))],
                             "BLS", grid=grid, domain="flux", workers=4)
    assert res.rows == [] and res.launches == 0
    assert set(res.errors) == {"star", "curve"}
    assert "no band has enough" in res.errors["star"]
    assert res.errors["curve"].startswith("InsufficientDataError")


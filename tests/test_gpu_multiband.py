"""Multi-band BLS on the engine -- the independent stack and the joint
(shared-box) search -- against the reference's golden output
(tests/golden/make_golden_multiband.py) and the oracle's joint sweep."""

from __future__ import annotations

import numpy as np
import pytest

from test_multiband_host import _cases, mblc_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [c for c in _cases() if c[0]["ephemeris"] == "independent"],
                         ids=lambda c: c[0]["key"])
def test_multiband_matches_reference(case):
    from cuperiod_b200.api import periodogram
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    meta, z = case
    k = meta["key"]
    grid = GridSpec(kind="period", values=z[f"{k}_periods"]) if meta["explicit_grid"] else None
    mblc = mblc_of(meta, z)
    pg = periodogram(mblc, "BLS", grid=grid, settings=BLSSettings())
    assert list(pg.meta["bands"]) == meta["used_bands"]
    assert pg.meta["mb_ephemeris"] == "independent"
    assert pg.n_samples == meta["n_samples"] and pg.baseline == meta["baseline"]
    np.testing.assert_array_equal(pg.frequency, z[f"{k}_frequency"])
    ref = z[f"{k}_power"]
    # per-band powers within 1e-6 relative, so their quadrature stack too
    np.testing.assert_allclose(pg.power, ref, rtol=1e-6, atol=1e-9 * float(np.max(ref)))
    band = pg.extras["band_index"] == z[f"{k}_x_band_index"]
    assert band.mean() >= 0.99
    same = band & (pg.extras["duration"] == z[f"{k}_x_duration"])
    assert same.mean() >= 0.98
    np.testing.assert_allclose(pg.extras["depth"][same], z[f"{k}_x_depth"][same], rtol=1e-6,
                               atol=1e-12)
    np.testing.assert_allclose(pg.extras["sde"], z[f"{k}_x_sde"], rtol=1e-5, atol=1e-6)
    assert pg.best_period() == meta["best_period"]

"""TLS host logic against the reference's golden output and known answers (no
GPU): the default period grid, template widths, templates, settings bounds,
the constant-flux short cut and the method registry."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from test_oracle_tls import case_inputs, tls_cases


@pytest.mark.parametrize("case", [c for c in tls_cases() if c[0]["default_grid"]],
                         ids=lambda c: c[0]["key"])
def test_default_grid_matches_reference(case):
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import TLSMethod
    meta, z = case
    t, y, dy, periods, _ = case_inputs(meta, z)
    grid = TLSMethod().default_grid(LightCurve(t, y, dy, Domain.FLUX),
                                    TLSSettings(**meta["settings"]))
    np.testing.assert_array_equal(grid.period, periods)


def test_widths_and_templates_match_the_oracle():
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import duration_bins, limb_darkened_template
    s = TLSSettings()
    assert duration_bins(s) == [3, 5, 8, 14, 26]
    assert duration_bins(TLSSettings(n_phase_bins=16, duration_min_frac=1e-4,
                                     duration_max_frac=2e-4, n_durations=3)) == [1]
    for n in (1, 2, 3, 8, 26, 101):
        for u1, u2 in ((0.4, 0.3), (0.5, 0.2), (0.0, 0.0), (1.0, 0.0)):
            np.testing.assert_array_equal(limb_darkened_template(n, u1, u2),
                                          oracle.tls_template(n, u1, u2))


def test_settings_bounds():
    from cuperiod_b200.settings import TLSSettings
    with pytest.raises(ValueError, match="limb"):
        TLSSettings(limb_dark_u1=0.8, limb_dark_u2=0.3)
    with pytest.raises(ValueError):
        TLSSettings(min_period_days=5.0, max_period_days=2.0)
    with pytest.raises(ValueError):
        TLSSettings(n_phase_bins=8)


def test_constant_flux_needs_no_device():
    # a constant flux finds no dip anywhere: zeros and t0 = t.min() (tls.py:681-682)
    from cuperiod_b200.settings import TLSSettings
    from cuperiod_b200.tls import tls_power
    t = np.linspace(3.0, 20.0, 300)
    out = tls_power(t, np.full(300, 7.0), None, np.geomspace(1.0, 5.0, 40),
                    settings=TLSSettings())
    for k in ("sde", "sr", "depth", "duration"):
        assert np.all(out[k] == 0.0)
    assert np.all(out["t0"] == 3.0)


def test_registry_and_multiband_refusal():
    from cuperiod_b200 import get_method
    from cuperiod_b200.api import periodogram
    from cuperiod_b200.lightcurve import Domain, LightCurve
    assert get_method("tls").name == "TLS" and get_method("TLS").settings_cls.__name__ == \
        "TLSSettings"
    bands = {b: LightCurve(np.arange(30.0), np.ones(30), None, Domain.FLUX) for b in "gr"}
    with pytest.raises(ValueError, match="multi-band"):
        periodogram(bands, "TLS")


def test_shared_axis_periodograms_equal_from_spectrum():
    # power_many sorts the shared grid once; each periodogram must equal what
    # Periodogram.from_spectrum builds for that curve alone
    from cuperiod_b200.lightcurve import Domain, LightCurve
    from cuperiod_b200.tls import TLSMethod, period_grid
    from cuperiod_b200.settings import TLSSettings
    rng = np.random.default_rng(2)
    t = np.sort(rng.uniform(0.0, 40.0, 500))
    lc = LightCurve(t, 1.0 + 1e-3 * rng.normal(size=t.size), None, Domain.FLUX)
    periods = period_grid(lc.baseline, TLSSettings())
    res = {k: rng.normal(size=periods.size) for k in ("sde", "sr", "depth", "duration", "t0")}
    m = TLSMethod()
    a = m._periodogram(res, periods, lc)
    b = m._periodogram(res, periods, lc, m._sorted_axis(periods))
    for name in ("frequency", "period", "power"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name
    assert a.extras.keys() == b.extras.keys()
    assert all(np.array_equal(a.extras[k], b.extras[k]) for k in a.extras)
    assert (a.n_samples, a.baseline, dict(a.meta)) == (b.n_samples, b.baseline, dict(b.meta))

"""Host-side inputs of the device peak ranking (no device)."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("overrides", [{}, {"peak_separation_rayleigh": 3.0},
                                       {"alias_freq_tolerance": 2e-3, "harmonic_max": 4}])
def test_peak_params_are_the_per_curve_defaults(overrides):
    # the device ranking's separation and alias tolerance per curve equal the
    # defaults Periodogram.best_periods resolves curve by curve
    from cuperiod_b200.bls import _peak_params
    from cuperiod_b200.result import DEFAULT_HARMONIC_MAX, DEFAULT_SEPARATION_RAYLEIGH
    from cuperiod_b200.settings import BLSSettings, peak_defaults
    s = BLSSettings(**overrides)
    baselines = 10.0 ** np.random.default_rng(3).uniform(-1.0, 3.5, 200)
    order, sep, tol = _peak_params(baselines, s)
    d = peak_defaults(s)
    sep_r = float(d.get("min_separation_rayleigh", DEFAULT_SEPARATION_RAYLEIGH))
    assert order == int(d.get("harmonic_max", DEFAULT_HARMONIC_MAX))
    for b, got_sep, got_tol in zip(baselines.tolist(), sep, tol):
        separation = sep_r / b
        t = d.get("alias_tolerance")
        t = t if t is not None else min(separation, 1.0 / b)
        assert got_sep == max(separation, 1e-12)
        assert got_tol == max(float(t), 1e-12)

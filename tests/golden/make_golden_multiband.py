"""Generate multi-band BLS golden vectors from the reference's own numba backend.

Run once in a container that holds the reference source (the committed
``multiband_cases.npz``/``.json`` are what the tests read)::

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/numba-cache \\
        python tests/golden/make_golden_multiband.py

Each case is ``bls_multiband_power(grid, mblc, settings, "numba", BLSMethod(),
ephemeris=...)`` (``src/cuperiod/multiband/bls_mb.py:120-315``; the shared
ephemeris runs the joint sweep of ``src/cuperiod/multiband/_bls_joint.py:412-527``):
the bands' inputs, the grid (explicit, or the stacked-baseline default grid of
``src/cuperiod/api.py:195-200``), the ephemeris mode and objective, and the
periodogram (frequency, power, the extras with ``band_index``, the band names,
``n_samples``, ``baseline``, the best period).
"""

from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def band(n, *, span, period, depth, noise, level, seed, with_error=True, t0=0.37):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0.0, span, n)) + 2459000.0
    flux = level * (1.0 + rng.normal(0.0, noise, n))
    flux[np.mod(t - 2459000.0 - t0 * period, period) < 0.08] -= level * depth
    err = np.full(n, level * noise) * rng.uniform(0.8, 1.2, n) if with_error else None
    return t, flux, err


def cases():
    three = {
        "g": band(1500, span=60.0, period=3.1, depth=4e-3, noise=2e-3, level=1.0, seed=1),
        "r": band(1200, span=55.0, period=3.1, depth=4e-3, noise=3e-3, level=2.5, seed=2),
        "i": band(900, span=62.0, period=3.1, depth=4e-3, noise=5e-3, level=4.0, seed=3),
    }
    scatter = {
        "V": band(700, span=40.0, period=2.3, depth=6e-3, noise=3e-3, level=1.0, seed=4),
        "B": band(500, span=38.0, period=2.3, depth=6e-3, noise=4e-3, level=0.7, seed=5,
                  with_error=False),
    }
    dropped = {
        "a": band(800, span=30.0, period=1.9, depth=5e-3, noise=2e-3, level=1.0, seed=6),
        "b": band(2, span=30.0, period=1.9, depth=5e-3, noise=2e-3, level=1.0, seed=7),
        "c": band(600, span=31.0, period=1.9, depth=5e-3, noise=2e-3, level=1.3, seed=8),
    }
    yield "three_bands_errors", three, np.geomspace(0.8, 10.0, 4000), "independent", "snr"
    yield "robust_scatter_default_grid", scatter, None, "independent", "snr"
    yield "short_band_dropped", dropped, np.geomspace(0.7, 8.0, 3000), "independent", "snr"
    yield "shared_three_bands", three, np.geomspace(0.8, 10.0, 4000), "shared", "snr"
    yield "shared_default_grid", scatter, None, "shared", "snr"
    yield "shared_band_dropped_likelihood", dropped, np.geomspace(0.7, 8.0, 3000), "shared", \
        "likelihood"
    # Bands observed at different epochs: the later band's times start well after the
    # common origin, and one band never dips (its depth is zero).
    late = band(600, span=20.0, period=2.7, depth=5e-3, noise=2e-3, level=1.0, seed=9)
    flat = band(500, span=25.0, period=2.7, depth=0.0, noise=2e-3, level=3.0, seed=10)
    yield "shared_offset_epochs", {
        "early": band(700, span=20.0, period=2.7, depth=5e-3, noise=2e-3, level=1.0, seed=11),
        "late": (late[0] + 37.25, late[1], late[2]),
        "flat": (flat[0] + 11.5, flat[1], flat[2]),
    }, np.geomspace(0.6, 9.0, 3500), "shared", "snr"


def main() -> None:
    from cuperiod.api import _multiband_grid
    from cuperiod.core.config import BLSSettings
    from cuperiod.core.grid import GridSpec
    from cuperiod.core.lightcurve import LightCurve, MultiBandLightCurve
    from cuperiod.methods.bls import BLSMethod
    from cuperiod.multiband.bls_mb import bls_multiband_power

    method = BLSMethod()
    store, index = {}, []
    for name, bands, periods, ephemeris, objective in cases():
        settings = BLSSettings(objective=objective)
        mblc = MultiBandLightCurve.from_light_curves(
            {k: LightCurve.from_arrays(t, y, e, domain="flux") for k, (t, y, e) in bands.items()})
        grid = (GridSpec(kind="period", values=periods) if periods is not None
                else _multiband_grid(method, mblc, settings))
        pg = bls_multiband_power(grid, mblc, settings, "numba", method, ephemeris=ephemeris)
        assert pg.meta["mb_ephemeris"] == ephemeris
        for k, (t, y, e) in bands.items():
            store[f"{name}_{k}_t"] = t
            store[f"{name}_{k}_y"] = y
            if e is not None:
                store[f"{name}_{k}_dy"] = e
        store[f"{name}_periods"] = np.asarray(grid.period, dtype=np.float64)
        store[f"{name}_frequency"] = pg.frequency
        store[f"{name}_power"] = pg.power
        for k, v in pg.extras.items():
            store[f"{name}_x_{k}"] = np.asarray(v, dtype=np.float64)
        index.append({"key": name, "bands": list(bands), "with_error": [e is not None for _, _, e in bands.values()],
                      "explicit_grid": periods is not None, "ephemeris": ephemeris,
                      "objective": objective,
                      "grid_meta": {k: (list(v) if isinstance(v, tuple) else v)
                                    for k, v in dict(grid.meta).items()},
                      "used_bands": list(pg.meta["bands"]), "n_samples": pg.n_samples,
                      "baseline": pg.baseline, "best_period": pg.best_period(),
                      "extras": list(pg.extras)})
    np.savez_compressed(os.path.join(HERE, "multiband_cases.npz"), **store)
    with open(os.path.join(HERE, "multiband_cases.json"), "w") as fh:
        json.dump(index, fh, indent=1, default=float)


if __name__ == "__main__":
    main()

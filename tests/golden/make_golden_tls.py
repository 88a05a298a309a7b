"""Generate TLS golden vectors from the reference's own numba backend.

Run once in a container that holds the reference source (the committed
``tls_cases.npz``/``.json`` are what the tests read)::

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/numba-cache \\
        python tests/golden/make_golden_tls.py

Each case is ``tls_power(t, y, dy, periods, settings=..., backend="numba")``
(``src/cuperiod/methods/tls.py:624-755``) on a seeded light curve, over the
periods of ``TLSMethod().default_grid`` (``tls.py:772-779``) or an explicit
grid, with the settings' non-default fields recorded.
"""

from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def curve(seed, n, span, *, period, depth, noise, level=1.0, t_off=0.0, with_error=True,
          spread=0.2):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0.0, span, n)) + t_off
    y = level * (1.0 + rng.normal(0.0, noise, n))
    ph = np.mod(t - t_off - 0.3 * period, period) / period
    y[np.minimum(ph, 1.0 - ph) < 0.02] -= level * depth
    dy = level * noise * rng.uniform(1.0 - spread, 1.0 + spread, n) if with_error else None
    return t, y, dy


def cases():
    yield "errors_default_grid", curve(1, 3000, 40.0, period=3.3, depth=2e-3, noise=1e-3), \
        None, {}
    yield "no_errors_explicit_grid", curve(2, 1500, 25.0, period=1.7, depth=4e-3, noise=2e-3,
                                           level=1.3e4, with_error=False), \
        np.geomspace(0.6, 10.0, 2500), {"n_phase_bins": 512, "n_durations": 7,
                                        "limb_dark_u1": 0.5, "limb_dark_u2": 0.2}
    yield "offset_epoch_wide_errors", curve(3, 2200, 60.0, period=5.1, depth=1.5e-3,
                                            noise=8e-4, t_off=2459000.25, spread=0.9), \
        None, {"duration_min_frac": 0.02, "duration_max_frac": 0.15, "n_durations": 4}
    t = np.sort(np.random.default_rng(4).uniform(0.0, 20.0, 400))
    yield "constant_flux", (t, np.full(400, 2.5), np.full(400, 0.1)), \
        np.geomspace(0.7, 9.0, 300), {}


def main() -> None:
    from cuperiod.core.config import TLSSettings
    from cuperiod.core.lightcurve import LightCurve
    from cuperiod.methods.tls import TLSMethod, tls_power

    store, index = {}, []
    for name, (t, y, dy), periods, kw in cases():
        settings = TLSSettings(**kw)
        if periods is None:
            lc = LightCurve.from_arrays(t, y, dy, domain="flux")
            periods = TLSMethod().default_grid(lc, settings).period
        res = tls_power(t, y, dy, periods, settings=settings, backend="numba")
        store[f"{name}_t"] = t
        store[f"{name}_y"] = y
        if dy is not None:
            store[f"{name}_dy"] = dy
        store[f"{name}_periods"] = np.asarray(periods, dtype=np.float64)
        for k, v in res.items():
            store[f"{name}_{k}"] = np.asarray(v, dtype=np.float64)
        index.append({"key": name, "with_error": dy is not None, "settings": kw,
                      "default_grid": name.endswith("default_grid") or
                      name == "offset_epoch_wide_errors",
                      "outputs": sorted(res)})
    np.savez_compressed(os.path.join(HERE, "tls_cases.npz"), **store)
    with open(os.path.join(HERE, "tls_cases.json"), "w") as fh:
        json.dump(index, fh, indent=1)


if __name__ == "__main__":
    main()

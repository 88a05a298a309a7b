"""Generate the BLS golden vectors from the reference's own numba backend.

Run once in a container that holds the reference source (it is not needed
anywhere else; the committed ``.npz``/``.json`` files are what the tests read)::

    PYTHONPATH=<reference>/src NUMBA_CACHE_DIR=/tmp/numba-cache \\
        python tests/golden/make_golden.py

Every case stores its inputs and the reference's outputs:

* ``kernel_cases.npz`` -- ``bls_power(..., backend="numba")``
  (``src/cuperiod/methods/_bls_core.py:882-1028``) on eclipsers, the adversarial
  inputs of the reference's screen test, sparse-tie curves, half-bin durations and
  the single-curve 2000-point / 10,000-period likelihood workload.
* ``method_cases.npz`` + ``method_cases.json`` -- ``BLSMethod.power`` on default and
  custom grids (``src/cuperiod/methods/bls.py:361-395``): spectrum, extras, the
  best period and the alias-diverse peak list, and the batch row
  (``src/cuperiod/batch/io.py:507-571``).
* ``grid_cases.json`` -- default-grid sizes, segment metadata and a digest of the
  period values (``bls.py:52-125, 327-359``).
"""

from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def eclipser(*, n=800, span=200.0, period=2.5, depth=0.05, frac=0.04, epoch=2458000.3,
             noise=0.005, base=2458000.0, seed=1):
    """Sorted-uniform times with periodic box dips and Gaussian noise."""
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0.0, span, n)) + base
    phase = ((t - epoch) % period) / period
    flux = np.ones(n)
    flux[(phase < frac) | (phase > 1.0 - frac)] -= depth
    flux += rng.normal(0.0, noise, n)
    return t, flux, np.full(n, noise)


def single_curve_workload(seed=0):
    """2000 points over 90 d, 2e-3 transit at 3.7 d / 0.1 d, 1e-3 noise, unit weights."""
    rng = np.random.default_rng(seed)
    n = 2000
    t = np.sort(rng.uniform(0.0, 90.0, n))
    flux = 1.0 + rng.normal(0.0, 1e-3, n)
    t0 = rng.uniform(0.0, 1.0) * 3.7
    flux[np.mod(t - t0, 3.7) < 0.1] -= 2e-3
    return t, flux, np.ones(n)


def adversarial_cases():
    """Offsets, constant and quantised flux, wild and huge errors, extreme scales."""
    rng = np.random.default_rng(11)
    t, flux, err = eclipser(n=300, span=60.0)
    n = t.size
    cases = [
        ("eclipser", t, flux, err),
        ("offset 1e6", t, flux + 1e6, err),
        ("offset 1e9", t, flux + 1e9, err),
        ("constant", t, np.ones(n), err),
        ("quantised ties", t, rng.integers(0, 3, n) * 0.01, err),
        ("wild errors", t, flux, 10.0 ** rng.uniform(-3.0, 1.0, n)),
        ("five points", t[:: n // 5][:5], flux[:: n // 5][:5], err[:: n // 5][:5]),
        ("pure noise", t, 1.0 + err * rng.standard_normal(n), err),
        ("huge errors", t, flux, np.full(n, 1e150)),
        ("both x 1e-60", t, flux * 1e-60, err * 1e-60),
        ("both x 1e60", t, flux * 1e60, err * 1e60),
    ]
    for scale in (1e-140, 1e-158, 1e-200, 1e140, 1e160):
        cases.append((f"flux x {scale:g}", t, flux * scale, err))
    return cases


def sparse_curve(n):
    rng = np.random.default_rng(n)
    t = 2458000.0 + np.sort(rng.uniform(0.0, 90.0, n))
    flux = 1.0 + rng.normal(0.0, 0.005, n)
    flux[np.mod(t - 2458000.3, 2.5) < 0.1] -= 0.01
    return t, flux, np.full(n, 0.005)


def transit_curve(n=800, seed=2):
    rng = np.random.default_rng(seed)
    t = 2458000.0 + np.sort(rng.uniform(0.0, 60.0, n))
    flux = 1.0 + rng.normal(0.0, 0.002, n)
    flux[np.mod(t - 2458001.3, 3.7) / 3.7 < 0.03] -= 0.01
    return t, flux, np.full(n, 0.002)


def long_period_eclipser():
    rng = np.random.default_rng(4)
    t = np.sort(rng.uniform(0.0, 400.0, 3000)) + 2458000.0
    flux = 1.0 + 0.002 * rng.standard_normal(t.size)
    phase = ((t - 2458011.0) % 37.3) / 37.3
    flux[(phase < 0.45 / 37.3) | (phase > 1.0 - 0.45 / 37.3)] -= 0.01
    return t, flux, np.full(t.size, 0.002)


def two_runs(seed):
    rng = np.random.default_rng(seed)
    t = np.concatenate([np.sort(rng.uniform(0.0, 3.0, 150)),
                        np.sort(rng.uniform(365.0, 368.0, 150))]) + 2458000.0
    err = rng.uniform(0.003, 0.008, t.size)
    flux = 1.0 + err * rng.standard_normal(t.size)
    return t, flux, err


def main() -> None:
    import cuperiod as cup
    from cuperiod.batch.io import periodogram_to_row
    from cuperiod.core.grid import GridSpec, log_period_grid
    from cuperiod.methods._bls_core import bls_power
    from cuperiod.methods.bls import BLSMethod

    fields = ("power", "depth", "depth_err", "depth_snr", "duration", "transit_time",
              "log_likelihood")
    store: dict[str, np.ndarray] = {}
    index: list[dict] = []

    def kernel_case(name, t, y, dy, periods, durations, oversample, objective):
        key = f"k{len(index):03d}"
        with np.errstate(over="ignore"):
            out = bls_power(t, y, dy, periods, durations, oversample, objective=objective,
                            backend="numba")
        store[f"{key}_t"] = np.asarray(t, np.float64)
        store[f"{key}_y"] = np.asarray(y, np.float64)
        store[f"{key}_dy"] = np.asarray(dy, np.float64)
        store[f"{key}_periods"] = np.asarray(periods, np.float64)
        store[f"{key}_durations"] = np.asarray(durations, np.float64)
        store[f"{key}_out"] = np.stack([getattr(out, f) for f in fields])
        index.append({"key": key, "name": name, "oversample": int(oversample),
                      "objective": objective})

    t, f, e = eclipser()
    for obj in ("snr", "likelihood"):
        kernel_case(f"eclipser {obj}", t, f, e, np.linspace(1.5, 4.0, 400),
                    np.array([0.05, 0.1, 0.2]), 10, obj)
    t, f, e = single_curve_workload()
    kernel_case("single-curve 2000 pts x 10000 periods likelihood", t, f, e,
                np.geomspace(0.5, 30.0, 10000), np.array([0.05, 0.08, 0.12, 0.16, 0.2]),
                10, "likelihood")
    for name, t, y, dy in adversarial_cases():
        for obj in ("snr", "likelihood"):
            kernel_case(f"adversarial {name} {obj}", t, y, dy, np.linspace(0.6, 9.0, 160),
                        np.array([0.02, 0.05, 0.11, 0.3]), 3, obj)
    for n in (45, 300):
        t, f, e = sparse_curve(n)
        kernel_case(f"sparse ties n={n}", t, f, e, np.linspace(1.0, 6.0, 1000),
                    np.geomspace(0.02, 0.4, 6), 5, "snr")
    t, f, e = eclipser()
    for durs in ((0.2, 0.25), (0.2, 0.45)):
        kernel_case(f"half-bin durations {durs}", t, f, e, np.linspace(1.5, 4.0, 300),
                    np.array(durs), 2, "snr")
    rng = np.random.default_rng(0)
    t = np.sort(rng.uniform(0.0, 27.0, 6000)) + 2458000.0
    flux = 1.0 + 1e-4 * rng.standard_normal(t.size)
    flux[((t - 2458000.4) % 3.1) / 3.1 < 0.03] -= 3e-4
    kernel_case("ppm photometry", t, flux, np.full(t.size, 1e-4), np.linspace(2.5, 4.0, 300),
                np.array([0.05, 0.1, 0.15]), 10, "snr")
    t, f, _ = eclipser(n=200)
    kernel_case("every weight underflows", t, f, np.full(t.size, 1e200),
                np.linspace(0.6, 9.0, 160), np.array([0.02, 0.05, 0.11, 0.3]), 3, "snr")
    np.savez_compressed(os.path.join(HERE, "kernel_cases.npz"), **store)
    with open(os.path.join(HERE, "kernel_cases.json"), "w") as fh:
        json.dump(index, fh, indent=1)

    # --- method-level: grid + segments + assemble + peaks + batch row ---------------
    method = BLSMethod()
    mstore: dict[str, np.ndarray] = {}
    mindex: list[dict] = []

    def method_case(name, t, flux, err, settings_kw, grid_kind, grid_kw=None):
        key = f"m{len(mindex):03d}"
        settings = cup.BLSSettings(**settings_kw)
        lc = cup.LightCurve.from_arrays(t, flux, err, domain=cup.Domain.FLUX)
        if grid_kind == "default":
            grid = method.default_grid(lc, settings)
        else:
            grid = log_period_grid(**grid_kw)
        pg = method.power(grid, lc, settings, "numba").with_peak_defaults(settings)
        mstore[f"{key}_t"] = np.asarray(t, np.float64)
        mstore[f"{key}_flux"] = np.asarray(flux, np.float64)
        mstore[f"{key}_err"] = np.asarray(err, np.float64)
        mstore[f"{key}_grid"] = np.asarray(grid.period, np.float64)
        mstore[f"{key}_frequency"] = pg.frequency
        mstore[f"{key}_power"] = pg.power
        for k, v in pg.extras.items():
            mstore[f"{key}_x_{k}"] = v
        peaks = pg.best_periods(10, alias_diverse=True)
        row = periodogram_to_row(name, pg, n_best=10, store_raw=False, alias_diverse=True)
        mindex.append({
            "key": key, "name": name, "settings": settings_kw,
            "grid_meta": {k: (list(v) if isinstance(v, tuple) else v)
                          for k, v in grid.meta.items()},
            "best_period": pg.best_period(),
            "peaks": [p.to_dict() for p in peaks],
            "row": {k: (None if isinstance(v, float) and np.isnan(v) else v)
                    for k, v in row.items()},
            "n_samples": pg.n_samples, "baseline": pg.baseline,
        })

    t, f, e = transit_curve()
    method_case("transit default grid", t, f, e,
                {"min_period_days": 0.5, "max_period_days": 10.0}, "default")
    method_case("transit default grid likelihood", t, f, e,
                {"min_period_days": 0.5, "max_period_days": 10.0, "objective": "likelihood"},
                "default")
    t, f, e = long_period_eclipser()
    method_case("long-period eclipser custom log grid", t, f, e, {}, "log",
                {"minimum_period": 1.0, "maximum_period": 100.0, "n_periods": 4000})
    for seed in (1, 5):
        t, f, e = two_runs(seed)
        method_case(f"two runs seed {seed} likelihood", t, f, e,
                    {"objective": "likelihood", "min_period_days": 20.0}, "default")
    t, f, e = eclipser(span=80.0)
    method_case("eclipser narrow default grid", t, f, e,
                {"min_period_days": 2.0, "max_period_days": 3.0}, "default")
    np.savez_compressed(os.path.join(HERE, "method_cases.npz"), **mstore)
    with open(os.path.join(HERE, "method_cases.json"), "w") as fh:
        json.dump(mindex, fh, indent=1, default=float)

    # --- default grids ----------------------------------------------------------------
    gindex = []
    for baseline, kw in ((27.0, {}), (60.0, {}), (90.0, {"min_period_days": 0.5}),
                         (115.35, {}), (1461.0, {"n_durations": 12, "max_period_days": 400.0}),
                         (200.0, {"segment_factor": 3.0, "grid_oversample": 5})):
        settings = cup.BLSSettings(**kw)
        tt = np.linspace(0.0, baseline, 50) + 2458000.0
        lc = cup.LightCurve.from_arrays(tt, np.ones(tt.size), np.ones(tt.size),
                                        domain=cup.Domain.FLUX)
        grid = method.default_grid(lc, settings)
        per = np.ascontiguousarray(grid.period, dtype=np.float64)
        gindex.append({"baseline_input": [float(tt[0]), float(tt[-1]), int(tt.size)],
                       "settings": kw, "size": int(per.size),
                       "segment_starts": list(grid.meta["segment_starts"]),
                       "segment_sizes": list(grid.meta["segment_sizes"]),
                       "first": float(per[0]), "last": float(per[-1]),
                       "sha256": hashlib.sha256(per.tobytes()).hexdigest()})
    # the 50,000-period log grid of the batched workload: its segments
    per = np.geomspace(0.3, 13.0, 50000)
    from cuperiod.methods.bls import _grid_segments
    segs = _grid_segments(GridSpec(kind="period", values=per), cup.BLSSettings())
    gindex.append({"log_grid": [0.3, 13.0, 50000],
                   "segment_sizes": [int(p.size) for p, _ in segs],
                   "segment_durations": [d.tolist() for _, d in segs]})
    with open(os.path.join(HERE, "grid_cases.json"), "w") as fh:
        json.dump(gindex, fh, indent=1)
    print(f"{len(index)} kernel cases, {len(mindex)} method cases, {len(gindex)} grids",
          file=sys.stderr)


if __name__ == "__main__":
    main()

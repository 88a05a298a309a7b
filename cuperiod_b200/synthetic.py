"""Seeded synthetic light curves with the shapes of the BLS benchmark workloads.

No survey data is available offline, so these stand in for it with the stated
cadences, lengths and value distributions:

* :func:`batched_curves` -- light curves of N ~ U[500, 20000] points over a 27 d
  baseline at 2-minute cadence with a 1 d gap in the middle and 5% random
  dropouts; FP32 flux 1 + N(0, sigma), sigma log-uniform in [2e-4, 5e-3]; half
  of them carry box transits (depth log-uniform [1e-4, 1e-2], period log-uniform
  [0.5, 13] d, duration U[0.02, 0.25] d); no errors (one weight per curve), or
  per-point errors sigma x U(0.7, 1.4).  Searched over 50,000
  log-spaced periods in [0.3, 13] d with the default 8 durations per segment.
* :func:`proposal_curves` -- training curves of the period-proposal network:
  the same cadence and noise, 60% with box transits, 40% noise (half with a
  sinusoid of amplitude log-uniform in [1e-4, 1e-2], period log-uniform in
  [0.1, 20] d).
* :func:`catalogue_curves` -- a packed catalogue for the streamed sweep:
  lognormal point counts (median 3000, 200-60,000), mixed 2-minute / 27 d and
  30-minute / 4-year cadences, half with box transits.
* :func:`single_curve` -- 2000 points uniform over 90 d, a 2e-3 transit at 3.7 d
  lasting 0.1 d, 1e-3 noise, unit errors; 10,000 log periods in [0.5, 30] d with
  durations {0.05, 0.08, 0.12, 0.16, 0.2} d and the likelihood objective.
* :func:`long_baseline_curves` -- 60,000 points at 30-minute cadence over four
  years with times offset by ~1.4e3 d, depths down to 5e-5; 200,000 log periods
  in [0.5, 400] d with 12 durations per segment.
* :func:`multiband_stars` -- stars observed in six bands (u, g, r, i, z, y; the
  points of a star split 6/9/26/26/17/16% between them) at random night-time
  epochs over 90 d, N ~ U[600, 3000] points per star; per band a flux level
  log-uniform in [0.3, 3], noise sigma log-uniform in [1e-3, 1e-2] with errors
  of sigma x U[0.8, 1.2]; half the stars carry a chromatic box transit (depth
  log-uniform [1e-3, 1e-2] scaled 0.7-1.3x from u to y, period log-uniform
  [0.5, 20] d, duration U[0.04, 0.3] d).  Searched with the shared box over the
  default grid of the stacked baseline.
* :func:`tls_curves` -- Kepler-like long-cadence light curves for the TLS
  search: a 30-minute cadence over 625 d, N ~ U[10000, 30000] points kept at
  random (the first and last always, so every curve has the same baseline and
  default grid), flux 1 + N(0, sigma), sigma log-uniform in [1e-4, 1e-3], errors
  sigma x U[0.9, 1.1]; half carry a box transit (period log-uniform [0.5, 12] d,
  duration U[0.05, 0.3] d, depth log-uniform [1e-4, 3e-3]).  Searched over
  0.5-12 d on the default TLS grid.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Curve:
    t: np.ndarray
    y: np.ndarray
    dy: np.ndarray | None
    transit: tuple[float, float, float] | None     # (period, duration, depth)


def _box(t, rng, period, duration, depth, y):
    t0 = rng.uniform(0.0, period)
    y[np.mod(t - t0, period) < duration] -= depth


def batched_curves(n_curves: int, *, seed: int = 0, n_range=(500, 20000),
                   weights: str = "uniform") -> list[Curve]:
    """The batched workload's light curves (see the module docstring).  Flux is
    rounded to FP32 (survey photometry is stored in single precision).
    ``weights="hetero"`` gives every point an error sigma x U(0.7, 1.4) (per-point
    photometric errors) instead of none."""
    rng = np.random.default_rng(seed)
    cadence = 2.0 / 1440.0
    base = np.arange(0.0, 27.0, cadence)
    base = base[(base < 13.0) | (base >= 14.0)]            # 1 d mid-baseline gap
    out = []
    for _ in range(n_curves):
        keep = base[rng.random(base.size) > 0.05]          # 5% dropouts
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        if keep.size > n:
            keep = np.sort(rng.choice(keep, n, replace=False))
        sigma = 10.0 ** rng.uniform(np.log10(2e-4), np.log10(5e-3))
        y = 1.0 + rng.normal(0.0, sigma, keep.size)
        transit = None
        if rng.random() < 0.5:
            period = 10.0 ** rng.uniform(np.log10(0.5), np.log10(13.0))
            duration = rng.uniform(0.02, 0.25)
            depth = 10.0 ** rng.uniform(-4.0, -2.0)
            _box(keep, rng, period, duration, depth, y)
            transit = (period, duration, depth)
        dy = None
        if weights == "hetero":
            dy = sigma * rng.uniform(0.7, 1.4, keep.size)
        y = y.astype(np.float32).astype(np.float64)
        out.append(Curve(keep + 2460000.0, y, dy, transit))
    return out


def proposal_curves(n_curves: int, *, seed: int = 0, n_range=(500, 20000)) -> list[Curve]:
    """Training curves of the period-proposal network: the batched workload's
    cadence, lengths and noise, with box transits (as there) on 60% of the
    curves; the other 40% are noise, half of them with a sinusoid of amplitude
    log-uniform in [1e-4, 1e-2] and period log-uniform in [0.1, 20] d."""
    rng = np.random.default_rng(seed)
    cadence = 2.0 / 1440.0
    base = np.arange(0.0, 27.0, cadence)
    base = base[(base < 13.0) | (base >= 14.0)]
    out = []
    for _ in range(n_curves):
        keep = base[rng.random(base.size) > 0.05]
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        if keep.size > n:
            keep = np.sort(rng.choice(keep, n, replace=False))
        sigma = 10.0 ** rng.uniform(np.log10(2e-4), np.log10(5e-3))
        y = 1.0 + rng.normal(0.0, sigma, keep.size)
        transit = None
        if rng.random() < 0.6:
            period = 10.0 ** rng.uniform(np.log10(0.5), np.log10(13.0))
            duration = rng.uniform(0.02, 0.25)
            depth = 10.0 ** rng.uniform(-4.0, -2.0)
            _box(keep, rng, period, duration, depth, y)
            transit = (period, duration, depth)
        elif rng.random() < 0.5:
            amp = 10.0 ** rng.uniform(-4.0, -2.0)
            ps = 10.0 ** rng.uniform(-1.0, np.log10(20.0))
            y += amp * np.sin(2.0 * np.pi * keep / ps + rng.uniform(0.0, 2.0 * np.pi))
        out.append(Curve(keep + 2460000.0, y.astype(np.float32).astype(np.float64), None,
                         transit))
    return out


def catalogue_curves(n_curves: int, *, seed: int = 0):
    """A catalogue of light curves, packed: ``(t, y, offsets, kind)`` with curve c
    at ``[offsets[c], offsets[c + 1])`` of the FP64 arrays ``t`` and ``y`` (FP32
    flux values).  Point counts are lognormal (median 3000, clipped to
    200-60,000); cadences are mixed: ``kind`` 0 is the batched workload's 2-minute
    cadence over 27 d (5% dropouts, a 1 d gap), ``kind`` 1 the long-baseline
    workload's 30-minute cadence over four years (two curves in ten); noise
    sigma log-uniform in [2e-4, 5e-3]; half carry box transits (depth log-uniform
    [1e-4, 1e-2], period log-uniform [0.5, 13] d, duration U[0.02, 0.25] d).  A
    curve's count is capped at its cadence's samples."""
    rng = np.random.default_rng(seed)
    short = np.arange(0.0, 27.0, 2.0 / 1440.0)
    short = short[(short < 13.0) | (short >= 14.0)]
    long_ = np.arange(60000) * (30.0 / 1440.0)
    long_ = long_ * (1461.0 / long_[-1])
    ts, ys, sizes = [], [], np.empty(n_curves, dtype=np.int64)
    kind = (rng.random(n_curves) < 0.2).astype(np.int8)
    for c in range(n_curves):
        base = long_ if kind[c] else short
        keep = base[rng.random(base.size) > 0.05]
        n = int(np.clip(np.exp(rng.normal(np.log(3000.0), 0.8)), 200, 60000))
        if keep.size > n:
            keep = np.sort(rng.choice(keep, n, replace=False))
        sigma = 10.0 ** rng.uniform(np.log10(2e-4), np.log10(5e-3))
        y = 1.0 + rng.normal(0.0, sigma, keep.size)
        if rng.random() < 0.5:
            period = 10.0 ** rng.uniform(np.log10(0.5), np.log10(13.0))
            _box(keep, rng, period, rng.uniform(0.02, 0.25), 10.0 ** rng.uniform(-4.0, -2.0), y)
        ts.append(keep + (2460000.0 if not kind[c] else 1400.0))
        ys.append(y.astype(np.float32).astype(np.float64))
        sizes[c] = keep.size
    offsets = np.zeros(n_curves + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    return np.concatenate(ts), np.concatenate(ys), offsets, kind


def batched_periods() -> np.ndarray:
    """50,000 log-spaced trial periods over [0.3, 13] d."""
    return np.geomspace(0.3, 13.0, 50000)


def single_curve(seed: int = 0) -> Curve:
    """The single-curve workload's light curve."""
    rng = np.random.default_rng(seed)
    n = 2000
    t = np.sort(rng.uniform(0.0, 90.0, n))
    y = 1.0 + rng.normal(0.0, 1e-3, n)
    t0 = rng.uniform(0.0, 1.0) * 3.7
    y[np.mod(t - t0, 3.7) < 0.1] -= 2e-3
    return Curve(t, y, np.ones(n), (3.7, 0.1, 2e-3))


SINGLE_PERIODS = (0.5, 30.0, 10000)
SINGLE_DURATIONS = (0.05, 0.08, 0.12, 0.16, 0.2)


def long_baseline_curves(n_curves: int, *, seed: int = 0) -> list[Curve]:
    """The long-baseline precision workload's light curves."""
    rng = np.random.default_rng(seed)
    t = np.arange(60000) * (30.0 / 1440.0)                 # 30-min cadence, 1250 d
    t = t * (1461.0 / t[-1]) + 1400.0                      # four years, offset ~1.4e3 d
    out = []
    for _ in range(n_curves):
        sigma = 10.0 ** rng.uniform(np.log10(2e-4), np.log10(5e-3))
        y = 1.0 + rng.normal(0.0, sigma, t.size)
        period = 10.0 ** rng.uniform(np.log10(0.5), np.log10(400.0))
        duration = rng.uniform(0.02, 0.25)
        depth = 10.0 ** rng.uniform(np.log10(5e-5), -2.0)
        _box(t, rng, period, duration, depth, y)
        # FP32 flux, transits included (the photometry is stored in single precision)
        y = y.astype(np.float32).astype(np.float64)
        out.append(Curve(t.copy(), y, None, (period, duration, depth)))
    return out


def long_baseline_periods() -> np.ndarray:
    """200,000 log-spaced trial periods over [0.5, 400] d."""
    return np.geomspace(0.5, 400.0, 200000)


MULTIBAND_BANDS = ("u", "g", "r", "i", "z", "y")
MULTIBAND_SHARE = (0.06, 0.09, 0.26, 0.26, 0.17, 0.16)


def multiband_stars(n_stars: int, *, seed: int = 0, span: float = 90.0,
                    n_range=(600, 3000)) -> list[dict[str, Curve]]:
    """The multi-band workload's stars, ``{band: Curve}`` each (see the module
    docstring)."""
    rng = np.random.default_rng(seed)
    stars = []
    for _ in range(n_stars):
        n_total = int(rng.integers(n_range[0], n_range[1] + 1))
        transit = None
        if rng.random() < 0.5:
            transit = (10.0 ** rng.uniform(np.log10(0.5), np.log10(20.0)),
                       rng.uniform(0.04, 0.3), 10.0 ** rng.uniform(-3.0, -2.0))
            t0 = rng.uniform(0.0, transit[0])
        bands = {}
        for b, (name, share) in enumerate(zip(MULTIBAND_BANDS, MULTIBAND_SHARE)):
            n = max(3, int(round(n_total * share)))
            nights = rng.integers(0, int(span), size=n)
            t = np.sort(nights + rng.uniform(0.05, 0.45, size=n)) + 2460000.0
            level = 10.0 ** rng.uniform(np.log10(0.3), np.log10(3.0))
            sigma = 10.0 ** rng.uniform(-3.0, -2.0)
            y = level * (1.0 + rng.normal(0.0, sigma, n))
            if transit is not None:
                scale = 0.7 + 0.6 * b / (len(MULTIBAND_BANDS) - 1)
                y[np.mod(t - 2460000.0 - t0, transit[0]) < transit[1]] -= \
                    level * transit[2] * scale
            dy = level * sigma * rng.uniform(0.8, 1.2, n)
            bands[name] = Curve(t, y, dy, transit)
        stars.append(bands)
    return stars


def tls_curves(n_curves: int, *, seed: int = 0, n_range=(10000, 30000)) -> list[Curve]:
    """The TLS workload's light curves (see the module docstring)."""
    rng = np.random.default_rng(seed)
    base = np.arange(30000) * (30.0 / 1440.0)               # 625 d at 30-minute cadence
    out = []
    for _ in range(n_curves):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        inner = rng.choice(np.arange(1, base.size - 1), n - 2, replace=False)
        t = base[np.sort(np.concatenate([[0, base.size - 1], inner]))] + 2454964.5
        sigma = 10.0 ** rng.uniform(-4.0, -3.0)
        y = 1.0 + rng.normal(0.0, sigma, t.size)
        transit = None
        if rng.random() < 0.5:
            period = 10.0 ** rng.uniform(np.log10(0.5), np.log10(12.0))
            duration = rng.uniform(0.05, 0.3)
            depth = 10.0 ** rng.uniform(-4.0, np.log10(3e-3))
            _box(t, rng, period, duration, depth, y)
            transit = (period, duration, depth)
        out.append(Curve(t, y, sigma * rng.uniform(0.9, 1.1, t.size), transit))
    return out


__all__ = ["Curve", "MULTIBAND_BANDS", "batched_curves", "batched_periods", "catalogue_curves",
           "proposal_curves",
           "long_baseline_curves", "long_baseline_periods", "multiband_stars", "single_curve",
           "tls_curves"]

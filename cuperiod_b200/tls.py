"""Transit least squares on the B200 engine (cuPeriod src/cuperiod/methods/tls.py).

A limb-darkened matched filter: per trial period the flux is folded into
``n_phase_bins`` phase bins and a quadratic limb-darkening template, resampled
to each trial width, is slid over every start phase; at each position the level
and the depth are fitted jointly by weighted least squares, and the signal
residue ``SR = (sum w g y')^2 / D`` with ``D = sum w g^2 - (sum w g)^2 / W`` is
kept where the fit is a dip.  The per-period maximum is normalised over the grid
into the SDE.

The host steps before and after the kernel are the reference's own numpy
operations (constant-flux test, power-of-two flux scale, weights, weighted mean,
templates, SDE and unit conversions), so the engine receives exactly what the
reference's kernel receives; the kernel (``bls_tls_search``) runs on the GPU.
There is no CPU fallback.
"""

from __future__ import annotations

import math
from typing import Any, ClassVar, Final, Literal, Sequence

import numpy as np

from . import _lib
from .errors import BackendUnavailableError, InsufficientDataError
from .grid import GridSpec, check_grid_size
from .lightcurve import Domain, LightCurve
from .result import Periodogram
from .settings import TLSSettings

BACKEND_NAME: Final = "b200"
BACKENDS: Final = frozenset({"auto", "gpu", "cupy", "cuda", "b200"})

W_EPS: Final = 1e-300               # smallest admissible template energy (tls.py:57)
DEN_REL_EPS: Final = 1e-9           # relative floor of D in float64 (tls.py:63)
CONSTANT_ULPS: Final = 64.0         # a flux within this many ulps is constant (tls.py:68)
OUTPUTS: Final = ("sde", "sr", "depth", "duration", "t0")


def limb_darkened_template(n: int, u1: float, u2: float) -> np.ndarray:
    """The peak-normalised flux deficit of a central transit over ``n`` samples
    under quadratic limb darkening ``I(mu) = 1 - u1 (1 - mu) - u2 (1 - mu)^2``
    (tls.py:84-111)."""
    if n <= 1:
        return np.ones(max(n, 1), dtype=np.float64)
    x = (np.arange(n, dtype=np.float64) + 0.5) / n - 0.5
    z = np.clip(2.0 * np.abs(x), 0.0, 1.0)
    mu = np.sqrt(1.0 - z * z)
    g = 1.0 - u1 * (1.0 - mu) - u2 * (1.0 - mu) ** 2
    g = np.where(z < 1.0, g, 0.0)
    peak = float(g.max())
    return g / peak if peak > 0.0 else g


def duration_bins(settings: TLSSettings) -> list[int]:
    """Template widths in bins, deduplicated and ascending, clamped to
    ``[1, n_bins - 1]`` (tls.py:114-126)."""
    n_bins = settings.n_phase_bins
    fracs = np.geomspace(settings.duration_min_frac, settings.duration_max_frac,
                         settings.n_durations)
    return sorted({min(max(int(round(f * n_bins)), 1), n_bins - 1) for f in fracs})


def grid_duration_frac(settings: TLSSettings) -> float:
    """The period grid's phase-drift budget: ``grid_duration_frac``, at most twice
    the shortest duration (tls.py:129-138)."""
    return min(settings.grid_duration_frac, 2.0 * settings.duration_min_frac)


def period_grid(baseline: float, settings: TLSSettings, *,
                time: np.ndarray | None = None) -> np.ndarray:
    """Ascending trial periods of a frequency grid capped by the baseline; the
    size is checked before allocating (tls.py:141-170)."""
    max_period = min(settings.max_period_days, baseline / settings.min_transits)
    if max_period <= settings.min_period_days:
        return np.zeros(0, dtype=np.float64)
    df = grid_duration_frac(settings) / (settings.oversample * baseline)
    f_lo, f_hi = 1.0 / max_period, 1.0 / settings.min_period_days
    check_grid_size(math.ceil((f_hi - f_lo) / df), automatic=True, time=time,
                    baseline=baseline,
                    context="TLS default period grid (min_period_days, grid_duration_frac "
                            "and oversample set its size)")
    freq = np.arange(f_lo, f_hi, df)
    if freq.size == 0:
        return np.zeros(0, dtype=np.float64)
    return np.ascontiguousarray(1.0 / freq[::-1], dtype=np.float64)


def is_constant(y: np.ndarray) -> bool:
    """Constant to within CONSTANT_ULPS ulps of its largest magnitude (tls.py:187-198)."""
    if y.size == 0:
        return True
    scale = float(np.max(np.abs(y)))
    return float(np.ptp(y)) <= CONSTANT_ULPS * float(np.finfo(np.float64).eps) * scale


def flux_scale(y: np.ndarray, dy: np.ndarray | None) -> float:
    """A power of two near the flux noise (median |dy|, else std y), so weights
    stay in range in any flux unit; dividing by it is exact (tls.py:201-212)."""
    s = float(np.std(y)) if dy is None else float(np.median(np.abs(dy)))
    if not (math.isfinite(s) and s > 0.0):
        return 1.0
    return 2.0 ** min(max(round(math.log2(s)), -1000), 1000)


def _no_transit(n_periods: int, t_ref: float) -> dict[str, np.ndarray]:
    out = {key: np.zeros(n_periods, dtype=np.float64) for key in OUTPUTS}
    out["t0"] = np.full(n_periods, t_ref, dtype=np.float64)
    return out


def _prepare(t, y, dy):
    """tls_power's host steps (tls.py:678-699): ``(kernel inputs or None,
    t_ref, scale)``."""
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    t_ref = float(t.min())
    if is_constant(y):
        return None, t_ref, 1.0
    scale = flux_scale(y, dy)
    y = y / scale
    w = (np.ones_like(y) if dy is None
         else 1.0 / (np.ascontiguousarray(dy, dtype=np.float64) / scale) ** 2)
    w_total = float(w.sum())
    y_mean = float(np.dot(w, y) / w_total)
    yw = w * (y - y_mean)
    return (t - t_ref, yw, w, w_total), t_ref, scale


def _finish(res: dict[str, np.ndarray], dy, t_ref: float, scale: float) -> dict[str, np.ndarray]:
    """SDE, flux units and absolute epochs (tls.py:737-755)."""
    sr = res["sr"]
    mean, std = float(sr.mean()), float(sr.std())
    res["sde"] = (sr - mean) / std if std > 0.0 else np.zeros_like(sr)
    res["depth"] = res["depth"] * scale
    if dy is None:
        res["sr"] = sr * (scale * scale)
    res["t0"] = res["t0"] + t_ref
    return res


def tls_power_many(curves: Sequence[tuple], periods, *, settings: TLSSettings,
                   engine: _lib.Engine | None = None) -> list[dict[str, np.ndarray]]:
    """``tls_power`` of many ``(t, y, dy or None)`` curves over one period grid,
    every searchable curve in one launch."""
    periods = np.ascontiguousarray(periods, dtype=np.float64)
    n_p = int(periods.size)
    if n_p == 0:
        return [{k: np.zeros(0) for k in OUTPUTS} for _ in curves]
    dur = duration_bins(settings)
    prepared = [_prepare(t, y, dy) for t, y, dy in curves]
    live = [i for i, (inp, _, _) in enumerate(prepared) if inp is not None and dur]
    results: list[dict[str, np.ndarray] | None] = [None] * len(curves)
    for i, (inp, t_ref, _) in enumerate(prepared):
        if inp is None or not dur:
            results[i] = _no_transit(n_p, t_ref)
    if live:
        u1, u2 = settings.limb_dark_u1, settings.limb_dark_u2
        templates = {wd: limb_darkened_template(wd, u1, u2) for wd in dur}
        out = (engine or _lib.default_engine()).tls_search(
            [prepared[i][0] for i in live], periods, n_bins=settings.n_phase_bins,
            dur_bins=dur, templates=templates, den_rel=DEN_REL_EPS)
        for j, i in enumerate(live):
            # views of the downloaded block (_finish replaces, never writes, them)
            res = {name: out[f, j] for f, name in enumerate(_lib.TLS_FIELD_NAMES)}
            results[i] = _finish(res, curves[i][2], prepared[i][1], prepared[i][2])
    return results  # type: ignore[return-value]


def tls_power(t, y, dy, periods, *, settings: TLSSettings,
              engine: _lib.Engine | None = None) -> dict[str, np.ndarray]:
    """The TLS search of one flux curve (tls.py:624-755): ``sde``, ``sr``,
    ``depth``, ``duration`` and ``t0`` (the mid-transit time of the first
    transit at or after ``t.min()``) per period; no dip anywhere (a constant
    flux) gives zeros and ``t0 = t.min()``."""
    return tls_power_many([(t, y, dy)], periods, settings=settings, engine=engine)[0]


class TLSMethod:
    """Transit Least Squares on the B200 engine (the reference's ``TLSMethod``,
    tls.py:758-826, with ``"b200"`` as its only backend)."""

    name: ClassVar[str] = "TLS"
    objective_sense: ClassVar[Literal["max", "min"]] = "max"
    supports_multiband: ClassVar[bool] = False
    natural_domain: ClassVar[Domain] = Domain.FLUX
    settings_cls: ClassVar[type] = TLSSettings
    gpu_backend: ClassVar[str] = BACKEND_NAME
    all_backends: ClassVar[tuple[str, ...]] = (BACKEND_NAME,)

    def resolve_backend(self, backend: str | None) -> str:
        b = (backend or "auto").lower()
        if b in BACKENDS:
            return BACKEND_NAME
        raise BackendUnavailableError(
            f"TLS backend {backend!r} is not available: this engine runs on the B200 only")

    def default_grid(self, lc: LightCurve, settings: TLSSettings) -> GridSpec:
        finite = lc.finite()
        periods = period_grid(finite.baseline, settings, time=finite.time)
        if periods.size == 0:
            raise InsufficientDataError("TLS: baseline too short for the configured period range")
        return GridSpec(kind="period", values=periods, uniform=False)

    def _checked(self, lc: LightCurve, settings: TLSSettings) -> LightCurve:
        finite = lc.finite()
        if finite.n < settings.min_detections:
            raise InsufficientDataError(
                f"TLS: {finite.n} finite points < min_detections {settings.min_detections}")
        if finite.baseline <= 0.0:
            raise InsufficientDataError("TLS: no usable time baseline")
        return finite

    def _periodogram(self, res, periods, finite: LightCurve, axis=None) -> Periodogram:
        """``axis``: ``(frequency, period, order)`` of the grid sorted into
        ascending frequency once for many curves (``_sorted_axis``)."""
        extras = {"sr": res["sr"], "depth": res["depth"], "duration": res["duration"],
                  "t0": res["t0"]}
        if axis is None:
            return Periodogram.from_spectrum(method="TLS", backend=BACKEND_NAME,
                                             frequency=1.0 / periods, power=res["sde"],
                                             objective_sense="max", n_samples=finite.n,
                                             baseline=finite.baseline, extras=extras,
                                             meta=finite.meta)
        frequency, period, order = axis
        return Periodogram("TLS", BACKEND_NAME, frequency, period,
                           np.ascontiguousarray(res["sde"][order]), "max", int(finite.n),
                           float(finite.baseline),
                           {k: np.ascontiguousarray(np.asarray(v, dtype=np.float64)[order])
                            for k, v in extras.items()}, dict(finite.meta or {}), {})

    @staticmethod
    def _sorted_axis(periods):
        """The grid in ascending frequency as ``Periodogram.from_spectrum`` sorts
        it, once: shared read-only frequency and period arrays and the order."""
        frequency = 1.0 / np.asarray(periods, dtype=np.float64)
        step = np.diff(frequency)
        if frequency.size < 2 or bool(np.all(step > 0.0)):
            order = slice(None)
        elif bool(np.all(step < 0.0)):
            order = slice(None, None, -1)
        else:
            order = np.argsort(frequency, kind="stable")
        frequency = np.ascontiguousarray(frequency[order])
        with np.errstate(divide="ignore"):
            period = 1.0 / frequency
        frequency.setflags(write=False)
        period.setflags(write=False)
        return frequency, period, order

    def power(self, grid: GridSpec, lc: LightCurve, settings: TLSSettings,
              backend: str = BACKEND_NAME, engine: _lib.Engine | None = None) -> Periodogram:
        """One light curve (tls.py:781-820)."""
        self.resolve_backend(backend)
        finite = self._checked(lc, settings)
        periods = grid.period
        res = tls_power(finite.time, finite.value, finite.error, periods, settings=settings,
                        engine=engine)
        return self._periodogram(res, periods, finite)

    def power_many(self, grid: GridSpec, lcs: Sequence[LightCurve], settings: TLSSettings,
                   backend: str = BACKEND_NAME, engine: _lib.Engine | None = None
                   ) -> list[Periodogram]:
        """Many light curves over one grid in one launch; one Periodogram each."""
        self.resolve_backend(backend)
        finite = [self._checked(lc, settings) for lc in lcs]
        periods = grid.period
        res = tls_power_many([(f.time, f.value, f.error) for f in finite], periods,
                             settings=settings, engine=engine)
        axis = self._sorted_axis(periods)
        return [self._periodogram(r, periods, f, axis) for r, f in zip(res, finite)]


def _register() -> None:
    from .bls import register
    register(TLSMethod())


_register()

__all__ = ["TLSMethod", "duration_bins", "limb_darkened_template", "period_grid", "tls_power",
           "tls_power_many"]

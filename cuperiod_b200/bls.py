"""The BLS method plugin on the B200 engine.

Mirrors cuPeriod's ``BLSMethod`` (src/cuperiod/methods/bls.py): the same
default log-segmented period grid, the same per-segment duration sets and the
same segmentation of custom grids, so the engine searches exactly the
(period, duration) trials the reference searches; ``power`` runs every segment
of a light curve in one engine launch and assembles the reference's
``Periodogram`` (SDE, extras, ascending frequency).  ``power_many`` searches a
whole chunk of light curves sharing one grid in one launch -- the hook the
batch runner uses instead of a per-curve loop.
"""

from __future__ import annotations

import functools
import math
from typing import Any, ClassVar, Literal, Sequence

import numpy as np

from . import _lib
from .core import BACKENDS, _objective_flag
from .errors import InsufficientDataError
from .grid import GridSpec, check_grid_size
from .lightcurve import Domain, LightCurve
from .result import Periodogram
from .settings import BLSSettings

#: Per-period fields of a segment (bls.py:33).
SEGMENT_FIELDS = ("period", "power", "depth", "depth_snr", "duration", "transit_time")

Segment = tuple[np.ndarray, np.ndarray]

#: The backend name recorded in results.
BACKEND_NAME = "b200"


def _segment_durations(p_lo: float, settings: BLSSettings) -> np.ndarray:
    """Box durations of the segment starting at ``p_lo`` (bls.py:39-49), read-only
    and shared: default grids of every baseline start their segments at the same
    ``min_period_days * segment_factor**k``, so a catalogue reuses a few arrays."""
    return _durations(float(p_lo), float(settings.duration_max_frac),
                      float(settings.duration_min_frac), float(settings.min_duration_days),
                      int(settings.n_durations))


@functools.lru_cache(maxsize=4096)
def _durations(p_lo: float, max_frac: float, min_frac: float, min_days: float,
               n: int) -> np.ndarray:
    d_hi = max_frac * p_lo
    d_lo = max(min_frac * p_lo, min_days)
    out = (np.asarray([d_hi], dtype=np.float64) if d_lo >= d_hi
           else np.asarray(np.geomspace(d_lo, d_hi, n), dtype=np.float64))
    out.setflags(write=False)
    return out


def _max_period(baseline: float, settings: BLSSettings) -> float:
    """Largest searchable period (bls.py:52-54)."""
    return min(settings.max_period_days, baseline / settings.min_transits)


def _segment_bounds(baseline: float, settings: BLSSettings) -> list[tuple[float, float]]:
    """``[(p_lo, p_hi), ...]`` of the default log segments (bls.py:57-68)."""
    max_period = _max_period(baseline, settings)
    bounds: list[tuple[float, float]] = []
    p_lo = settings.min_period_days
    while p_lo < max_period:
        p_hi = min(p_lo * settings.segment_factor, max_period)
        bounds.append((p_lo, p_hi))
        p_lo = p_hi
    return bounds


def _segment_periods(baseline: float, settings: BLSSettings, *, time=None,
                     context: str = "BLS default grid") -> list[tuple[float, np.ndarray]]:
    """Non-empty default segments, each uniform in frequency (bls.py:71-105)."""
    bounds = _segment_bounds(baseline, settings)
    if not bounds:
        return []
    df = settings.grid_duration_frac / (settings.grid_oversample * baseline)
    total = sum(max(0, math.ceil((1.0 / p_lo - 1.0 / p_hi) / df)) for p_lo, p_hi in bounds)
    check_grid_size(total, automatic=True, time=time, baseline=baseline, context=context)
    parts: list[tuple[float, np.ndarray]] = []
    for p_lo, p_hi in bounds:
        freq = np.arange(1.0 / p_hi, 1.0 / p_lo, df)
        freq = freq[freq < 1.0 / p_lo]   # arange may overshoot its stop by a rounding quantum
        if freq.size:
            parts.append((p_lo, np.asarray(1.0 / freq[::-1], dtype=np.float64)))
    return parts


def _default_total(baseline: float, settings: BLSSettings) -> int:
    """The size the reference checks before building a default grid (bls.py:81-84)."""
    bounds = _segment_bounds(baseline, settings)
    if not bounds:
        return 0
    df = settings.grid_duration_frac / (settings.grid_oversample * baseline)
    return sum(max(0, math.ceil((1.0 / p_lo - 1.0 / p_hi) / df)) for p_lo, p_hi in bounds)


def default_grid_spec(settings: BLSSettings, max_baseline: float) -> _lib.DefaultGridSpec:
    """The default grid's parameters for the engine library's host builder, with
    the box durations of every segment start that a baseline up to
    ``max_baseline`` reaches (starts min_period_days * segment_factor**k, as
    _segment_bounds steps them)."""
    max_period = _max_period(max_baseline, settings)
    durations = []
    p_lo = settings.min_period_days
    while p_lo < max_period:
        durations.append(_segment_durations(p_lo, settings))
        p_lo = p_lo * settings.segment_factor
    offsets = np.zeros(len(durations) + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([d.size for d in durations]) if durations else []
    return _lib.DefaultGridSpec(
        settings.min_period_days, settings.max_period_days, settings.min_transits,
        settings.segment_factor, settings.grid_duration_frac, settings.grid_oversample,
        offsets, np.ascontiguousarray(np.concatenate(durations) if durations else np.empty(0),
                                      dtype=np.float64),
        settings.bins_per_duration, _objective_flag(settings.objective))


def _segment_grids(baseline: float, settings: BLSSettings, *, time=None,
                   context: str = "BLS default grid") -> list[Segment]:
    """``[(periods, durations), ...]`` of the default grid (bls.py:108-125)."""
    return [(periods, _segment_durations(p_lo, settings))
            for p_lo, periods in _segment_periods(baseline, settings, time=time,
                                                  context=context)]


def _log_segments(periods: np.ndarray, settings: BLSSettings) -> list[Segment]:
    """Split any period grid into the default grid's log segments (bls.py:128-152)."""
    p0 = float(periods.min())
    with np.errstate(divide="ignore", invalid="ignore"):
        index = np.floor(np.log(periods / p0) / math.log(settings.segment_factor)
                         + 1e-9).astype(np.int64)
    return [(np.ascontiguousarray(periods[index == k]),
             _segment_durations(p0 * settings.segment_factor ** k, settings))
            for k in np.unique(index).tolist()]


def _grid_segments(grid: GridSpec, settings: BLSSettings) -> list[Segment]:
    """The segments that search exactly ``grid``'s periods (bls.py:155-190)."""
    periods = np.asarray(grid.period, dtype=np.float64)
    if periods.size == 0:
        return []
    if not np.all(np.isfinite(periods)):
        raise ValueError("BLS: trial periods must be finite; drop frequency 0 from the grid")
    starts = grid.meta.get("segment_starts")
    sizes = grid.meta.get("segment_sizes")
    if (starts is not None and sizes is not None and len(starts) == len(sizes)
            and sum(int(s) for s in sizes) == periods.size):
        segments: list[Segment] = []
        offset = 0
        for p_lo, size in zip(starts, sizes):
            stop = offset + int(size)
            segments.append((periods[offset:stop], _segment_durations(float(p_lo), settings)))
            offset = stop
        return segments
    return _log_segments(periods, settings)


def _assemble(fields: dict[str, np.ndarray], n: int, baseline: float, meta: Any) -> Periodogram:
    """SDE and the Periodogram of one curve's concatenated segments (bls.py:274-301)."""
    power = np.nan_to_num(fields["power"], nan=0.0, posinf=0.0, neginf=0.0)
    mean, std = float(power.mean()), float(power.std())
    sde = (power - mean) / std if std > 0.0 else np.zeros_like(power)
    extras = {"depth": fields["depth"], "depth_snr": fields["depth_snr"],
              "duration": fields["duration"], "t0": fields["transit_time"], "sde": sde}
    return Periodogram.from_spectrum(method="BLS", backend=BACKEND_NAME,
                                     frequency=1.0 / fields["period"], power=power,
                                     objective_sense="max", n_samples=n, baseline=baseline,
                                     extras=extras, meta=meta)


def _prepared_curve(lc: LightCurve, settings: BLSSettings):
    """``finite()`` and the reference's guards (bls.py:369-380).  A curve without
    errors keeps ``None``: the engine then takes every point's ivar as 1, the
    reference's unit errors, without an array of ones being built and packed."""
    finite = lc.finite()
    if finite.n < settings.min_detections:
        raise InsufficientDataError(
            f"BLS: {finite.n} finite points < min_detections {settings.min_detections}")
    if finite.baseline <= 0.0:
        raise InsufficientDataError("BLS: no usable time baseline")
    return finite, finite.error


class BLSMethod:
    """Box Least Squares on the B200 engine (the reference's ``BLSMethod``,
    bls.py:304-417, with ``"b200"`` as its only backend)."""

    name: ClassVar[str] = "BLS"
    objective_sense: ClassVar[Literal["max", "min"]] = "max"
    supports_multiband: ClassVar[bool] = True
    natural_domain: ClassVar[Domain] = Domain.FLUX
    settings_cls: ClassVar[type] = BLSSettings
    gpu_backend: ClassVar[str] = BACKEND_NAME
    all_backends: ClassVar[tuple[str, ...]] = (BACKEND_NAME,)

    def resolve_backend(self, backend: str | None) -> str:
        """Every GPU-ish selector resolves to this engine; CPU backends do not exist
        here and raise (there is no CPU fallback)."""
        b = (backend or "auto").lower()
        if b in BACKENDS:
            return BACKEND_NAME
        from .errors import BackendUnavailableError
        raise BackendUnavailableError(
            f"BLS backend {backend!r} is not available: this engine runs on the B200 only")

    def default_grid(self, lc: LightCurve, settings: BLSSettings) -> GridSpec:
        """Log period segments up to min(max_period_days, baseline/min_transits),
        with the segmentation recorded in ``meta`` (bls.py:327-359)."""
        finite = lc.finite()
        parts = _segment_periods(finite.baseline, settings, time=finite.time)
        if not parts:
            raise InsufficientDataError("BLS: baseline too short for the configured period range")
        periods = np.concatenate([p for _, p in parts])
        return GridSpec(kind="period", values=periods, uniform=False,
                        meta={"segmented": True,
                              "segment_starts": tuple(float(p) for p, _ in parts),
                              "segment_sizes": tuple(int(p.size) for _, p in parts)})

    def power(self, grid: GridSpec, lc: LightCurve, settings: BLSSettings,
              backend: str = BACKEND_NAME, engine: _lib.Engine | None = None) -> Periodogram:
        """One light curve: every segment in one launch, then the reference's
        assembly (bls.py:361-395)."""
        self.resolve_backend(backend)
        finite, err = _prepared_curve(lc, settings)
        segments = _grid_segments(grid, settings)
        if not segments:
            raise InsufficientDataError("BLS: empty trial grid")
        out = self._search(segments, [(finite.time, finite.value, err)], settings, engine)
        fields = _fields(out[:, 0, :], segments)
        return _assemble(fields, finite.n, finite.baseline, finite.meta)

    def power_many(self, grid: GridSpec, lcs: Sequence[LightCurve], settings: BLSSettings,
                   backend: str = BACKEND_NAME, engine: _lib.Engine | None = None
                   ) -> list[Periodogram]:
        """Many light curves over one grid in one launch; one Periodogram each."""
        self.resolve_backend(backend)
        segments = _grid_segments(grid, settings)
        if not segments:
            raise InsufficientDataError("BLS: empty trial grid")
        prepared = [_prepared_curve(lc, settings) for lc in lcs]
        out = self._search(segments, [(f.time, f.value, e) for f, e in prepared], settings, engine)
        return [_assemble(_fields(out[:, i, :], segments), f.n, f.baseline, f.meta)
                for i, (f, _) in enumerate(prepared)]

    def multiband_power(self, grid: GridSpec, mblc: Any, settings: BLSSettings,
                        backend: str = BACKEND_NAME, engine: _lib.Engine | None = None, *,
                        ephemeris: str | None = None) -> Periodogram:
        """Multi-band BLS on a shared period grid (bls.py:397-411 ->
        multiband/bls_mb.py:120-275); all bands in one engine launch."""
        from .multiband import bls_multiband_power
        self.resolve_backend(backend)
        return bls_multiband_power(grid, mblc, settings, ephemeris=ephemeris, engine=engine)

    def rows_many(self, grid: GridSpec, keyed: Sequence[tuple[str, LightCurve]],
                  settings: BLSSettings, *, n_best: int = 10, extra_keys: Sequence[str] = (),
                  engine: _lib.Engine | None = None) -> list[dict]:
        """Result rows of many light curves over one grid with their peaks ranked
        on the device: what ``periodogram_to_row(pg.with_peak_defaults(settings),
        n_best=..., alias_diverse=True)`` gives for each curve's periodogram
        (batch/io.py:507-571, core/result.py:285-367), without bringing the
        spectra back.  ``extra_keys``: the per-peak extras every rank carries
        (NaN past the last peak)."""
        return self.rows_by_grid([(key, lc, grid) for key, lc in keyed], settings,
                                 n_best=n_best, extra_keys=extra_keys, engine=engine)

    def rows_by_grid(self, items: Sequence[tuple[str, LightCurve, GridSpec]],
                     settings: BLSSettings, *, n_best: int = 10,
                     extra_keys: Sequence[str] = (),
                     engine: _lib.Engine | None = None,
                     prefiltered: bool = False) -> list[dict]:
        """``rows_many`` for curves that each bring their own grid (the
        reference's batch searches every curve over its own default grid,
        batch/runner.py:187-250): every curve of ``items`` -- ``(key, curve,
        grid)``, equal grids passed as the same object -- in one launch, each
        over its grid, peaks ranked on the device.  Rows in ``items`` order.
        ``prefiltered``: the curves are ``finite()`` results that already passed
        the minimum-detection and baseline guards (the batch runner's check), so
        they are not filtered again."""
        count = max(int(n_best), 1)
        slot: dict[int, int] = {}
        grids: list[GridSpec] = []
        gidx = np.empty(len(items), dtype=np.int32)
        for i, (_, _, g) in enumerate(items):
            k = slot.setdefault(id(g), len(grids))
            if k == len(grids):
                grids.append(g)
            gidx[i] = k
        segments = [_grid_segments(g, settings) for g in grids]
        if any(not sg for sg in segments):
            raise InsufficientDataError("BLS: empty trial grid")
        prepared = ([(lc, lc.error) for _, lc, _ in items] if prefiltered
                    else [_prepared_curve(lc, settings) for _, lc, _ in items])
        eng = engine or _lib.default_engine()
        periods = [np.concatenate([np.asarray(p, dtype=np.float64) for p, _ in sg])
                   for sg in segments]
        device_ok = [count <= 1024 and p.size >= 1 and bool(np.all(np.diff(p) > 0.0))
                     for p in periods]
        rows: list[dict | None] = [None] * len(items)
        host = [i for i in range(len(items)) if not device_ok[gidx[i]]]
        if host:
            # outside the device ranking's preconditions: rank on the host
            from .batch import periodogram_to_row
            for k in sorted({int(gidx[i]) for i in host}):
                members = [i for i in host if gidx[i] == k]
                out = self._search(segments[k], [(prepared[i][0].time, prepared[i][0].value,
                                                  prepared[i][1]) for i in members],
                                   settings, eng)
                for j, i in enumerate(members):
                    f = prepared[i][0]
                    rows[i] = periodogram_to_row(
                        items[i][0], _assemble(_fields(out[:, j, :], segments[k]), f.n,
                                               f.baseline, f.meta).with_peak_defaults(settings),
                        n_best=count, extra_keys=extra_keys, alias_diverse=True)
        dev = [i for i in range(len(items)) if device_ok[gidx[i]]]
        if dev:
            used = sorted({int(gidx[i]) for i in dev})
            local = {k: j for j, k in enumerate(used)}
            flag = _objective_flag(settings.objective)
            packed_grids = [_lib.PackedGrid.from_segments(segments[k], settings.bins_per_duration,
                                                          flag) for k in used]
            eng.prepare_grids(packed_grids, [local[int(gidx[i])] for i in dev],
                              _lib.PackedCurves.from_arrays(
                                  [(prepared[i][0].time, prepared[i][0].value, prepared[i][1])
                                   for i in dev]))
            eng.launch()
            base = [prepared[i][0].baseline for i in dev]
            order, sep, tol = _peak_params(base, settings)
            n_peaks, _, fields = eng.rows(count, order, sep, tol)
            made = self._rows([items[i][0] for i in dev], [prepared[i][0].n for i in dev], base,
                              n_peaks, fields, n_best, extra_keys)
            for j, i in enumerate(dev):
                rows[i] = made[j]
        return rows  # type: ignore[return-value]

    def split_default(self, keyed: Sequence[tuple[str, LightCurve]], settings: BLSSettings,
                      prefiltered: bool = False
                      ) -> tuple[list[tuple[str, LightCurve]], dict[str, str]]:
        """The curves whose default grid can be searched, and the failure of each
        other curve as ``default_grid`` would raise it (the grid-size guard,
        GridTooLargeError, or an empty grid, InsufficientDataError), without
        building the grids in Python (``prefiltered`` as in ``rows_by_grid``)."""
        from .errors import CuPeriodError
        good: list[tuple[str, LightCurve]] = []
        errors: dict[str, str] = {}
        base: list[float] = []
        for key, lc in keyed:
            finite = lc if prefiltered else lc.finite()
            b = finite.baseline
            try:
                check_grid_size(_default_total(b, settings), automatic=True, time=finite.time,
                                baseline=b, context="BLS default grid")
            except (CuPeriodError, ValueError) as exc:
                errors[key] = f"{type(exc).__name__}: {exc}"
                continue
            good.append((key, lc))
            base.append(b)
        if not good:
            return good, errors
        spec = default_grid_spec(settings, max(base))
        sizes = _lib.default_grid_sizes(spec, np.asarray(base))
        kept = []
        for (key, lc), n in zip(good, sizes):
            if n > 0:
                kept.append((key, lc))
            else:
                errors[key] = ("InsufficientDataError: BLS: baseline too short for the "
                               "configured period range")
        return kept, errors

    def rows_default(self, keyed: Sequence[tuple[str, LightCurve]], settings: BLSSettings, *,
                     n_best: int = 10, extra_keys: Sequence[str] = (),
                     engine: _lib.Engine | None = None,
                     prefiltered: bool = False) -> list[dict]:
        """``rows_by_grid`` with every curve over its own default grid
        (``default_grid``), the grids built by the engine library on the host
        cores (``bls_prepare_default``) instead of as one GridSpec per curve:
        the same trial periods bit for bit, the same rows.  The curves must pass
        ``split_default`` (``prefiltered`` as in ``rows_by_grid``)."""
        count = max(int(n_best), 1)
        if count > 1024:
            return self.rows_by_grid([(key, lc, self.default_grid(lc, settings))
                                      for key, lc in keyed], settings, n_best=n_best,
                                     extra_keys=extra_keys, engine=engine,
                                     prefiltered=prefiltered)
        prepared = ([(lc, lc.error) for _, lc in keyed] if prefiltered
                    else [_prepared_curve(lc, settings) for _, lc in keyed])
        if not prepared:
            return []
        baselines = np.array([f.baseline for f, _ in prepared], dtype=np.float64)
        spec = default_grid_spec(settings, float(baselines.max()))
        eng = engine or _lib.default_engine()
        eng.prepare_default(spec, baselines, _lib.PackedCurves.from_arrays(
            [(f.time, f.value, e) for f, e in prepared]))
        eng.launch()
        order, sep, tol = _peak_params(baselines, settings)
        n_peaks, _, fields = eng.rows(count, order, sep, tol)
        return self._rows([key for key, _ in keyed], [f.n for f, _ in prepared], baselines,
                          n_peaks, fields, n_best, extra_keys)

    def _rows(self, keys: Sequence[str], n_samples: Sequence[int], baselines: Sequence[float],
              n_peaks: np.ndarray, fields: np.ndarray, n_best: int,
              extra_keys: Sequence[str]) -> list[dict]:
        """The result rows from the device's ranked peaks (fields per rank:
        period, frequency, power, depth, depth_snr, duration, t0, sde): the
        reference's row layout (batch/io.py:507-571) -- best_period, then per
        rank period, power, the ``extra_keys`` (NaN where absent) and the other
        extras -- with the column names built once for all rows."""
        names = ("depth", "depth_snr", "duration", "t0", "sde")
        nan = float("nan")
        n_best = int(n_best)
        # per rank: period key, power key, the extra_keys' (key, field column or
        # None), the other extras' (key, column); a rank without a peak keeps
        # only the extra_keys, as NaN
        layout = []
        for rank in range(1, n_best + 1):
            asked = [(f"{e}_{rank}", 3 + names.index(e) if e in names else None)
                     for e in extra_keys]
            rest = [(f"{e}_{rank}", 3 + j) for j, e in enumerate(names) if e not in extra_keys]
            layout.append((f"period_{rank}", f"power_{rank}", asked, rest))
        counts = np.asarray(n_peaks).tolist()
        width = fields.shape[1]
        rows = []
        for j, key in enumerate(keys):
            k_have = int(counts[j])
            fl = fields[j, :min(k_have, width)].tolist()
            row: dict[str, Any] = {"key": key, "method": self.name, "backend": BACKEND_NAME,
                                   "n_samples": int(n_samples[j]),
                                   "baseline": float(baselines[j]),
                                   "best_period": fl[0][0] if k_have else nan}
            for r, (pk, wk, asked, rest) in enumerate(layout):
                if r < k_have:
                    fr = fl[r]
                    row[pk] = fr[0]
                    row[wk] = fr[2]
                    for ck, c in asked:
                        row[ck] = fr[c] if c is not None else nan
                    for ck, c in rest:
                        row[ck] = fr[c]
                else:
                    row[pk] = nan
                    row[wk] = nan
                    for ck, _ in asked:
                        row[ck] = nan
            rows.append(row)
        return rows

    def _search(self, segments, curves, settings, engine):
        grid = _lib.PackedGrid.from_segments(segments, settings.bins_per_duration,
                                             _objective_flag(settings.objective))
        packed = _lib.PackedCurves.from_arrays(curves)
        return (engine or _lib.default_engine()).search(grid, packed)


def _peak_params(baselines, settings: BLSSettings) -> tuple[int, np.ndarray, np.ndarray]:
    """The device ranking's inputs for curves of these baselines (all > 0):
    the harmonic order, and per curve the minimum frequency separation
    max(min_separation_rayleigh / baseline, 1e-12) and the alias tolerance
    max(alias_tolerance or min(separation, 1 / baseline), 1e-12) -- the
    defaults Periodogram.best_periods resolves (core/result.py:285-367)."""
    from .result import DEFAULT_HARMONIC_MAX, DEFAULT_SEPARATION_RAYLEIGH
    from .settings import peak_defaults
    d = peak_defaults(settings)
    sep_r = float(d.get("min_separation_rayleigh", DEFAULT_SEPARATION_RAYLEIGH))
    order = int(d.get("harmonic_max", DEFAULT_HARMONIC_MAX))
    tol_set = d.get("alias_tolerance")
    b = np.asarray(baselines, dtype=np.float64)
    separation = sep_r / b
    tol = (np.full(b.size, float(tol_set)) if tol_set is not None
           else np.minimum(separation, 1.0 / b))
    return order, np.maximum(separation, 1e-12), np.maximum(tol, 1e-12)


def _fields(out: np.ndarray, segments: list[Segment]) -> dict[str, np.ndarray]:
    """Engine rows (7, P) of one curve as the assembly's per-period fields."""
    names = _lib.FIELD_NAMES
    fields = {name: np.ascontiguousarray(out[i]) for i, name in enumerate(names)}
    fields["period"] = np.concatenate([np.asarray(p, dtype=np.float64) for p, _ in segments])
    return fields


_REGISTRY: dict[str, BLSMethod] = {}


def register(method: BLSMethod) -> None:
    _REGISTRY[method.name.upper()] = method


def get_method(name: str) -> BLSMethod:
    from .errors import UnknownMethodError
    key = "".join(ch for ch in str(name) if ch.isalnum()).upper()
    if key not in _REGISTRY:
        raise UnknownMethodError(f"unknown method {name!r}; this engine provides "
                                 f"{', '.join(sorted(_REGISTRY))}")
    return _REGISTRY[key]


register(BLSMethod())

__all__ = ["BLSMethod", "get_method", "register"]

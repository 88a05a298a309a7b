"""Result types of the BLS path: ``Peak`` and ``Periodogram`` with the
reference's peak selection (cuPeriod src/cuperiod/core/result.py:82-480 and
src/cuperiod/core/peaks.py:57-231)."""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Any, Literal, Mapping

import numpy as np

DEFAULT_N_PEAKS = 10
DEFAULT_SEPARATION_RAYLEIGH = 3.0
DEFAULT_HARMONIC_MAX = 8
PEAK_DEFAULT_FIELDS = ("n", "min_separation_rayleigh", "alias_tolerance", "harmonic_max",
                       "n_points")

SIDEREAL_FREQ_CPD = 1.0027379
SOLAR_FREQ_CPD = 1.0
YEARLY_FREQ_CPD = 1.0 / 365.25


def _interior_maxima(safe: np.ndarray) -> np.ndarray:
    """Strictly above the left neighbour, >= the right one (peaks.py:80-85)."""
    if safe.size < 3:
        return np.empty(0, dtype=np.int64)
    interior = (safe[1:-1] > safe[:-2]) & (safe[1:-1] >= safe[2:])
    return np.flatnonzero(interior).astype(np.int64) + 1


def select_top_peaks(frequency, score, candidates, n_peaks, min_separation) -> np.ndarray:
    """Greedy highest-score peaks at least ``min_separation`` apart (peaks.py:88-125)."""
    if n_peaks <= 0:
        return np.empty(0, dtype=np.int64)
    chosen: list[int] = []
    for idx in candidates[np.argsort(score[candidates])[::-1]]:
        if all(abs(frequency[idx] - frequency[j]) >= min_separation for j in chosen):
            chosen.append(int(idx))
            if len(chosen) >= n_peaks:
                break
    return np.asarray(chosen, dtype=np.int64)


def is_alias_related(f_new, f_chosen, tol, harmonic_max, *, min_separation=None) -> bool:
    """Duplicate, harmonic or daily/yearly alias of a chosen peak (peaks.py:128-180)."""
    separation = tol if min_separation is None else min_separation
    if abs(f_new - f_chosen) < separation:
        return True
    for m in range(2, harmonic_max + 1):
        if abs(f_new - m * f_chosen) < m * tol:
            return True
        if abs(f_new - f_chosen / m) < tol:
            return True
    offsets = [k * day for day in (SIDEREAL_FREQ_CPD, SOLAR_FREQ_CPD) for k in (1, 2)]
    offsets.append(YEARLY_FREQ_CPD)
    for off in offsets:
        if abs(f_new - abs(f_chosen - off)) < tol or abs(f_new - (f_chosen + off)) < tol:
            return True
    return False


def select_diverse_peaks(frequency, score, candidates, n_peaks, tol, harmonic_max, *,
                         min_separation=None) -> np.ndarray:
    """Greedy highest-score peaks skipping alias-related candidates (peaks.py:183-231)."""
    if n_peaks <= 0:
        return np.empty(0, dtype=np.int64)
    chosen: list[int] = []
    for idx in candidates[np.argsort(score[candidates])[::-1]]:
        f_new = float(frequency[idx])
        if all(not is_alias_related(f_new, float(frequency[j]), tol, harmonic_max,
                                    min_separation=min_separation)
               and not is_alias_related(float(frequency[j]), f_new, tol, harmonic_max,
                                        min_separation=min_separation)
               for j in chosen):
            chosen.append(int(idx))
            if len(chosen) >= n_peaks:
                break
    return np.asarray(chosen, dtype=np.int64)


@dataclass(frozen=True)
class Peak:
    """One periodogram peak (result.py:82-120)."""

    period: float
    frequency: float
    power: float
    rank: int
    extra: Mapping[str, float] = field(default_factory=dict, hash=False)

    def to_dict(self) -> dict:
        out = {"period": self.period, "frequency": self.frequency, "power": self.power,
               "rank": self.rank}
        out.update(self.extra)
        return out


@dataclass(frozen=True, eq=False)
class Periodogram:
    """A computed periodogram, sorted by ascending frequency (result.py:122-480)."""

    method: str
    backend: str
    frequency: np.ndarray
    period: np.ndarray
    power: np.ndarray
    objective_sense: Literal["max", "min"]
    n_samples: int
    baseline: float
    extras: Mapping[str, np.ndarray] = field(default_factory=dict)
    meta: Mapping[str, Any] = field(default_factory=dict)
    peak_defaults: Mapping[str, Any] = field(default_factory=dict)

    @classmethod
    def from_spectrum(cls, *, method, backend, frequency, power, objective_sense, n_samples,
                      baseline, extras=None, meta=None, peak_defaults=None) -> "Periodogram":
        """Stable-sort everything into ascending frequency (result.py:175-241)."""
        if objective_sense not in ("max", "min"):
            raise ValueError("objective_sense must be 'max' or 'min'")
        frequency = np.ascontiguousarray(frequency, dtype=np.float64)
        power = np.ascontiguousarray(power, dtype=np.float64)
        if frequency.ndim != 1 or power.shape != frequency.shape:
            raise ValueError("frequency must be 1-D and power of the same shape")
        # the stable sort of a strictly monotone grid (every grid built from
        # ascending periods) is the identity or a reversal: no gather needed
        step = np.diff(frequency)
        if frequency.size < 2 or bool(np.all(step > 0.0)):
            order: Any = slice(None)
        elif bool(np.all(step < 0.0)):
            order = slice(None, None, -1)
        else:
            order = np.argsort(frequency, kind="stable")
        frequency = np.ascontiguousarray(frequency[order])
        sorted_extras = {}
        for k, v in (extras or {}).items():
            arr = np.asarray(v, dtype=np.float64)
            if arr.shape != frequency.shape:
                raise ValueError(f"extras[{k!r}] shape does not match frequency")
            sorted_extras[k] = np.ascontiguousarray(arr[order])
        with np.errstate(divide="ignore"):
            period = 1.0 / frequency
        return cls(method, backend, frequency, period, np.ascontiguousarray(power[order]),
                   objective_sense, int(n_samples), float(baseline), sorted_extras,
                   dict(meta or {}), dict(peak_defaults or {}))

    def with_peak_defaults(self, defaults) -> "Periodogram":
        from .settings import peak_defaults as _from_settings
        new = dict(defaults) if isinstance(defaults, Mapping) else _from_settings(defaults)
        unknown = sorted(set(new) - set(PEAK_DEFAULT_FIELDS))
        if unknown:
            raise ValueError(f"unknown peak default(s) {unknown}")
        return dataclasses.replace(self, peak_defaults={**self.peak_defaults, **new})

    def _peak_default(self, name, fallback):
        value = self.peak_defaults.get(name)
        return fallback if value is None else value

    @property
    def size(self) -> int:
        return int(self.frequency.size)

    def _score(self) -> np.ndarray:
        return self.power if self.objective_sense == "max" else -self.power

    def _peak_candidates(self, score: np.ndarray) -> np.ndarray:
        """Interior local maxima plus boundary peaks over finite scores
        (result.py:369-406)."""
        usable = np.isfinite(score) & np.isfinite(self.period)
        safe = score if usable.all() else np.where(usable, score, -np.inf)
        candidates = _interior_maxima(safe)
        boundary: list[int] = []
        if self.size == 1:
            boundary.append(0)
        elif self.size >= 2:
            if safe[0] >= safe[1]:
                boundary.append(0)
            if safe[-1] > safe[-2]:
                boundary.append(self.size - 1)
        if boundary:
            candidates = np.concatenate([candidates, np.asarray(boundary, dtype=np.int64)])
        if candidates.size:
            ok = np.isfinite(score[candidates]) & np.isfinite(self.period[candidates])
            candidates = candidates[ok]
        if candidates.size == 0:
            finite = np.flatnonzero(usable)
            if finite.size == 0:
                return np.empty(0, dtype=np.int64)
            return finite[[int(np.argmax(score[finite]))]]
        return candidates

    def best_periods(self, n=None, *, min_separation_rayleigh=None, alias_diverse=False,
                     harmonic_max=None, alias_tolerance=None) -> list[Peak]:
        """The ``n`` most significant peaks (result.py:285-367)."""
        count = int(self._peak_default("n", DEFAULT_N_PEAKS)) if n is None else int(n)
        if count <= 0 or self.size == 0:
            return []
        score = self._score()
        candidates = self._peak_candidates(score)
        if candidates.size == 0:
            return []
        sep_r = float(self._peak_default("min_separation_rayleigh", DEFAULT_SEPARATION_RAYLEIGH)
                      if min_separation_rayleigh is None else min_separation_rayleigh)
        resolved = self.baseline > 0.0
        separation = sep_r / self.baseline if resolved else 0.0
        if alias_diverse:
            order = int(self._peak_default("harmonic_max", DEFAULT_HARMONIC_MAX)
                        if harmonic_max is None else harmonic_max)
            tol = self._peak_default("alias_tolerance", None) if alias_tolerance is None \
                else alias_tolerance
            if tol is None:
                tol = min(separation, 1.0 / self.baseline) if resolved else 0.0
            chosen = select_diverse_peaks(self.frequency, score, candidates, count,
                                          max(float(tol), 1e-12), order,
                                          min_separation=max(separation, 1e-12))
        else:
            chosen = select_top_peaks(self.frequency, score, candidates, count, separation)
        return [self._make_peak(int(i), rank) for rank, i in enumerate(chosen, 1)]

    def _make_peak(self, idx: int, rank: int) -> Peak:
        return Peak(float(self.period[idx]), float(self.frequency[idx]), float(self.power[idx]),
                    rank, {k: float(v[idx]) for k, v in self.extras.items()})

    def best_period(self) -> float:
        peaks = self.best_periods(1)
        return peaks[0].period if peaks else float("nan")


__all__ = ["Peak", "Periodogram", "is_alias_related", "select_diverse_peaks",
           "select_top_peaks"]

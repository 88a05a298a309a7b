"""Trial grids: ``GridSpec``, the size guard and the log-period grid
(cuPeriod src/cuperiod/core/grid.py:105-186, 417-505, 768-800)."""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field
from typing import Any, Literal, Mapping

import numpy as np

from .errors import GridTooLargeError

GridKind = Literal["frequency", "period"]

#: Hard ceiling on a trial grid's size (grid.py:57).
MAX_GRID_SIZE: int = 250_000_000
#: Automatic grids above this size warn and are still built (grid.py:62).
AUTO_GRID_WARN_SIZE: int = 5_000_000


class GridSizeWarning(UserWarning):
    """An automatic grid above :data:`AUTO_GRID_WARN_SIZE`."""


def _reciprocal_reversed(values: np.ndarray) -> np.ndarray:
    with np.errstate(divide="ignore"):
        return np.ascontiguousarray((1.0 / values)[::-1])


def _validate(values: np.ndarray, kind: str, uniform: bool) -> None:
    if values.size == 0:
        return
    if not np.all(np.isfinite(values)):
        raise ValueError("grid values must be finite")
    if kind == "frequency" and values.min() < 0.0:
        raise ValueError("frequency grid values must be >= 0")
    if kind == "period" and values.min() <= 0.0:
        raise ValueError("period grid values must be > 0")
    tol = 1e-9 * float(np.max(np.abs(values)))
    if values.size > 1 and np.any(np.diff(values) < -tol):
        raise ValueError("grid values must be ascending")
    if uniform:
        if kind != "frequency":
            raise ValueError("uniform=True requires a frequency grid")
        if values.size > 2:
            step = np.diff(values)
            if not np.allclose(step, step[0], rtol=1e-6, atol=0.0):
                raise ValueError("uniform=True but values are not an arithmetic progression")


@dataclass(frozen=True, eq=False)
class GridSpec:
    """A trial grid in the frequency or period domain (grid.py:105-186)."""

    kind: GridKind
    values: np.ndarray
    uniform: bool = False
    meta: Mapping[str, Any] = field(default_factory=dict)

    def __post_init__(self) -> None:
        if self.kind not in ("frequency", "period"):
            raise ValueError(f"grid kind must be 'frequency' or 'period', got {self.kind!r}")
        values = np.ascontiguousarray(np.asarray(self.values, dtype=np.float64))
        if values.ndim != 1:
            raise ValueError(f"grid values must be 1-D, got shape {values.shape}")
        _validate(values, self.kind, bool(self.uniform))
        object.__setattr__(self, "values", values)

    @property
    def size(self) -> int:
        return int(self.values.size)

    @property
    def frequency(self) -> np.ndarray:
        return self.values if self.kind == "frequency" else _reciprocal_reversed(self.values)

    @property
    def period(self) -> np.ndarray:
        return self.values if self.kind == "period" else _reciprocal_reversed(self.values)


def check_grid_size(n_points: int, *, limit: int | None = None, automatic: bool = False,
                    time: np.ndarray | None = None, baseline: float | None = None,
                    context: str = "trial grid") -> None:
    """Refuse a grid above the hard limit, warn about a large automatic grid
    (grid.py:417-505), before anything is allocated."""
    hard = MAX_GRID_SIZE if limit is None else int(limit)
    n_points = int(n_points)
    if n_points > hard:
        origin = f" over a {baseline:.6g}-day baseline" if baseline is not None else ""
        raise GridTooLargeError(
            f"{context}: {n_points:,} trial samples{origin} exceeds the limit of {hard:,}; "
            "check for mis-converted timestamps or pass an explicit grid=")
    if automatic and n_points > AUTO_GRID_WARN_SIZE:
        warnings.warn(GridSizeWarning(
            f"{context}: the automatic grid has {n_points:,} trial samples. Computing it anyway."),
            stacklevel=3)


def log_period_grid(*, minimum_period: float, maximum_period: float,
                    n_periods: int) -> GridSpec:
    """A log-spaced period grid (grid.py:768-800)."""
    if not (math.isfinite(minimum_period) and math.isfinite(maximum_period)):
        raise ValueError("minimum_period and maximum_period must be finite")
    if not 0.0 < minimum_period < maximum_period:
        raise ValueError("require 0 < minimum_period < maximum_period")
    if n_periods < 1:
        raise ValueError("n_periods must be >= 1")
    check_grid_size(n_periods, context="log_period_grid")
    return GridSpec(kind="period", values=np.geomspace(minimum_period, maximum_period, n_periods))


__all__ = ["AUTO_GRID_WARN_SIZE", "GridSizeWarning", "GridSpec", "MAX_GRID_SIZE",
           "check_grid_size", "log_period_grid"]

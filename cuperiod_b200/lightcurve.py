"""Light curves as the BLS path uses them (cuPeriod
src/cuperiod/core/lightcurve.py:230-303): finite-point filtering, the
magnitude-to-flux conversion and the baseline."""

from __future__ import annotations

from dataclasses import dataclass, field
from enum import Enum
from typing import Any, Mapping

import numpy as np


class Domain(str, Enum):
    """Brightness domain of a light curve's values."""

    MAGNITUDE = "magnitude"
    FLUX = "flux"


@dataclass(frozen=True, eq=False)
class LightCurve:
    """Times (days), values and optional 1-sigma errors of one band."""

    time: np.ndarray
    value: np.ndarray
    error: np.ndarray | None = None
    domain: Domain = Domain.MAGNITUDE
    meta: Mapping[str, Any] = field(default_factory=dict)

    def __post_init__(self) -> None:
        t = np.ascontiguousarray(self.time, dtype=np.float64).ravel()
        v = np.ascontiguousarray(self.value, dtype=np.float64).ravel()
        if t.shape != v.shape:
            raise ValueError("time and value must have the same length")
        object.__setattr__(self, "time", t)
        object.__setattr__(self, "value", v)
        if self.error is not None:
            e = np.ascontiguousarray(self.error, dtype=np.float64).ravel()
            if e.shape != t.shape:
                raise ValueError("error must have the length of time")
            object.__setattr__(self, "error", e)
        object.__setattr__(self, "domain", Domain(self.domain))

    @classmethod
    def from_arrays(cls, time, value, error=None, *, domain: Domain | str = Domain.MAGNITUDE,
                    meta: Mapping[str, Any] | None = None) -> "LightCurve":
        return cls(time, value, error, Domain(domain), dict(meta or {}))

    @property
    def n(self) -> int:
        return int(self.time.size)

    @property
    def baseline(self) -> float:
        return float(self.time.max() - self.time.min()) if self.n else 0.0

    def _usable(self) -> np.ndarray:
        mask = np.isfinite(self.time) & np.isfinite(self.value)
        if self.error is not None:
            mask &= np.isfinite(self.error) & (self.error > 0.0)
        return mask

    def finite(self) -> "LightCurve":
        """Drop non-finite points and non-positive errors (lightcurve.py:240-255)."""
        mask = self._usable()
        if mask.all():
            return self
        return LightCurve(self.time[mask], self.value[mask],
                          None if self.error is None else self.error[mask], self.domain, self.meta)

    def as_flux(self, *, zeropoint: float = 0.0) -> "LightCurve":
        """``flux = 10**(-0.4 (mag - zp))``, ``flux_err = 0.4 ln(10) flux mag_err``
        (lightcurve.py:257-267)."""
        if self.domain is Domain.FLUX:
            return self
        flux = np.power(10.0, -0.4 * (self.value - zeropoint))
        error = None if self.error is None else (0.4 * np.log(10.0)) * flux * self.error
        return LightCurve(self.time, flux, error, Domain.FLUX, self.meta)

    def in_domain(self, domain: Domain | str, *, zeropoint: float = 0.0) -> "LightCurve":
        if Domain(domain) is Domain.FLUX:
            return self.as_flux(zeropoint=zeropoint)
        if self.domain is Domain.MAGNITUDE:
            return self
        with np.errstate(invalid="ignore", divide="ignore"):
            mag = -2.5 * np.log10(self.value) + zeropoint
            err = None if self.error is None else (2.5 / np.log(10.0)) * self.error / self.value
        return LightCurve(self.time, mag, err, Domain.MAGNITUDE, self.meta)


__all__ = ["Domain", "LightCurve"]

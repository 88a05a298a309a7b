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


@dataclass(frozen=True, eq=False)
class MultiBandLightCurve:
    """Several bands (filters) of one star in one brightness domain
    (src/cuperiod/core/lightcurve.py:330-575); band order is insertion order."""

    bands: Mapping[str, LightCurve]
    meta: Mapping[str, Any] = field(default_factory=dict)

    def __post_init__(self) -> None:
        if not self.bands:
            raise ValueError("MultiBandLightCurve requires at least one band")
        for name, lc in self.bands.items():
            if not isinstance(lc, LightCurve):
                raise TypeError(f"band {name!r} is a {type(lc).__name__}, not a LightCurve")
        domains = {lc.domain for lc in self.bands.values()}
        if len(domains) > 1:
            listing = ", ".join(f"{k}: {lc.domain.value}" for k, lc in self.bands.items())
            raise ValueError(f"bands are in different brightness domains ({listing})")
        object.__setattr__(self, "bands", dict(self.bands))

    @classmethod
    def from_light_curves(cls, bands: Mapping[str, LightCurve], *,
                          meta: Mapping[str, Any] | None = None) -> "MultiBandLightCurve":
        return cls(dict(bands), dict(meta or {}))

    @property
    def band_names(self) -> tuple[str, ...]:
        return tuple(self.bands)

    @property
    def n_bands(self) -> int:
        return len(self.bands)

    def finite(self) -> "MultiBandLightCurve":
        """Each band's non-finite points removed (lightcurve.py:520-524)."""
        return MultiBandLightCurve({k: lc.finite() for k, lc in self.bands.items()}, self.meta)

    def stacked(self):
        """All bands in ascending time: ``(time, value, error or None, band)``;
        ``error`` is None when a band has none (lightcurve.py:544-575)."""
        times, values, errors, labels = [], [], [], []
        missing = False
        for name, lc in self.bands.items():
            times.append(lc.time)
            values.append(lc.value)
            if lc.error is None:
                missing = True
            else:
                errors.append(lc.error)
            labels.append(np.full(lc.n, name, dtype=object))
        time = np.concatenate(times)
        value = np.concatenate(values)
        band = np.concatenate(labels)
        error = None if missing else np.concatenate(errors)
        order = np.argsort(time, kind="stable")
        return time[order], value[order], None if error is None else error[order], band[order]


__all__ = ["Domain", "LightCurve", "MultiBandLightCurve"]

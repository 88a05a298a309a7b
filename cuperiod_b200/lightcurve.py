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

    @classmethod
    def from_dataframe(cls, df: Any, *, columns: Any = None, domain: Domain | str | None = None,
                       meta: Mapping[str, Any] | None = None) -> "LightCurve":
        """From a pandas/pyarrow/``{column: array}`` table with column detection
        (lightcurve.py:143-158)."""
        from .tables import adapt_table
        names, getter = adapt_table(df)
        return cls._from_table(names, getter, columns, domain, meta)

    @classmethod
    def from_file(cls, path: Any, *, columns: Any = None, domain: Domain | str | None = None,
                  meta: Mapping[str, Any] | None = None) -> "LightCurve":
        """From a CSV/TSV/ECSV/text/Parquet file with column detection; the
        format follows the extension (lightcurve.py:160-176)."""
        from .tables import adapt_table, read_table_object
        names, getter = adapt_table(read_table_object(path))
        return cls._from_table(names, getter, columns, domain,
                               {"source": str(path), **dict(meta or {})})

    @classmethod
    def _from_table(cls, names, getter, columns, domain, meta) -> "LightCurve":
        import warnings
        from .columns import ColumnMap
        from .tables import band_codes
        resolved = (columns or ColumnMap()).resolve(names, domain=domain)
        if resolved.band is not None:
            _, labels = band_codes(getter(resolved.band))
            if len(labels) > 1:
                warnings.warn(f"band column {resolved.band!r} holds {len(labels)} bands that "
                              "are pooled into one light curve; read the table as a "
                              "MultiBandLightCurve to keep them apart", UserWarning,
                              stacklevel=3)
        return cls._from_resolved(getter, resolved, meta)

    @classmethod
    def _from_resolved(cls, getter, resolved, meta) -> "LightCurve":
        from .tables import as_float
        return cls(as_float(getter(resolved.time)), as_float(getter(resolved.value)),
                   None if resolved.error is None else as_float(getter(resolved.error)),
                   resolved.domain, dict(meta or {}))

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

    def unusable_reason(self) -> str | None:
        """Why the errors leave no usable point, or ``None`` when they do not
        (lightcurve.py:306-326).  ``finite`` drops every point whose error is
        non-finite or ``<= 0``, so a placeholder error column (all 0, -1 or NaN)
        empties the curve; this names that cause.  ``None`` when there are no
        errors, when a point survives, or when no point has a finite time and
        value (a different problem, left to the caller)."""
        if self.error is None:
            return None
        data = np.isfinite(self.time) & np.isfinite(self.value)
        n_data = int(np.count_nonzero(data))
        if n_data == 0 or self._usable().any():
            return None
        return (f"none of the {n_data} points with a finite time and value has a usable "
                "error (all are zero, negative or non-finite), so every point would be "
                "dropped; drop the error column (error=None) to run unweighted")

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

    @classmethod
    def from_dataframe(cls, df: Any, *, band_column: str | None = None, columns: Any = None,
                       domain: Domain | str | None = None,
                       meta: Mapping[str, Any] | None = None) -> "MultiBandLightCurve":
        """From one long-format table split on its band column (lightcurve.py:389-425)."""
        return cls._from_table_object(df, band_column, columns, domain, meta)

    @classmethod
    def from_file(cls, path: Any, *, band_column: str | None = None, columns: Any = None,
                  domain: Domain | str | None = None,
                  meta: Mapping[str, Any] | None = None) -> "MultiBandLightCurve":
        """From one long-format table file split on its band column
        (lightcurve.py:427-463)."""
        from .tables import read_table_object
        return cls._from_table_object(read_table_object(path), band_column, columns, domain,
                                      {"source": str(path), **dict(meta or {})})

    @classmethod
    def _from_table_object(cls, table, band_column, columns, domain,
                           meta) -> "MultiBandLightCurve":
        """Rows without a band label are dropped; each band keeps its rows' order
        (lightcurve.py:465-518)."""
        import dataclasses
        import warnings
        from .columns import ColumnMap
        from .errors import ColumnResolutionError
        from .tables import adapt_table, band_codes
        names, getter = adapt_table(table)
        cmap = columns or ColumnMap(band=band_column)
        if band_column is not None and cmap.band is None:
            cmap = dataclasses.replace(cmap, band=band_column)
        resolved = cmap.resolve(names, domain=domain)
        if resolved.band is None:
            raise ColumnResolutionError("could not resolve a band column; pass band_column=... "
                                        f"or ColumnMap(band=...). Available columns: {names}")
        codes, labels = band_codes(getter(resolved.band))
        if not labels:
            raise ColumnResolutionError(f"band column {resolved.band!r} holds no labels")
        missing = int(np.count_nonzero(codes < 0))
        if missing:
            warnings.warn(f"{missing} of {codes.size} rows have no label in band column "
                          f"{resolved.band!r} and were dropped", UserWarning, stacklevel=3)
        whole = LightCurve._from_resolved(getter, resolved, None)
        order = np.argsort(codes, kind="stable")
        bounds = np.searchsorted(codes[order], np.arange(len(labels) + 1))
        time, value = whole.time[order], whole.value[order]
        error = None if whole.error is None else whole.error[order]
        bands = {}
        for k, label in enumerate(labels):
            rows = slice(int(bounds[k]), int(bounds[k + 1]))
            bands[label] = LightCurve(time[rows], value[rows],
                                      None if error is None else error[rows], whole.domain,
                                      {"band": label})
        return cls(bands, dict(meta or {}))

    @property
    def band_names(self) -> tuple[str, ...]:
        return tuple(self.bands)

    @property
    def n_bands(self) -> int:
        return len(self.bands)

    def finite(self) -> "MultiBandLightCurve":
        """Each band's non-finite points removed (lightcurve.py:520-524)."""
        return MultiBandLightCurve({k: lc.finite() for k, lc in self.bands.items()}, self.meta)

    def unusable_reason(self) -> str | None:
        """Why the errors leave no usable point in any band, or ``None``
        (lightcurve.py:526-542): each band whose error column is unusable is
        named, and only when no band keeps a point."""
        reasons: dict[str, str] = {}
        for name, lc in self.bands.items():
            reason = lc.unusable_reason()
            if reason is not None:
                reasons[name] = reason
            elif lc._usable().any():
                return None
        if not reasons:
            return None
        return "; ".join(f"band {name!r}: {why}" for name, why in reasons.items())

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


def raise_if_unusable(data: "LightCurve | MultiBandLightCurve", label: str) -> None:
    """Raise ``InsufficientDataError(f"{label}: {reason}")`` when an unusable error
    column would empty ``data`` (lightcurve.py:625-646).  Called before a grid is
    built, so the cause is named instead of surfacing as "no usable time
    baseline" from the emptied curve."""
    from .errors import InsufficientDataError
    reason = data.unusable_reason()
    if reason is not None:
        raise InsufficientDataError(f"{label}: {reason}")


__all__ = ["Domain", "LightCurve", "MultiBandLightCurve", "raise_if_unusable"]

"""Single-curve entry point: ``periodogram`` (cuPeriod src/cuperiod/api.py:204-307)
for the BLS method on the B200 engine."""

from __future__ import annotations

from typing import Any, Mapping

import numpy as np

from .bls import get_method
from .grid import GridSpec
from .lightcurve import Domain, LightCurve, MultiBandLightCurve
from .result import Periodogram
from .settings import BLSSettings


def to_input(data: Any, *, domain: Domain | str | None = None) -> LightCurve | MultiBandLightCurve:
    """A ``LightCurve`` from a LightCurve or a ``(t, y[, dy])`` tuple; a bare tuple
    is read as magnitudes unless ``domain`` says otherwise.  A MultiBandLightCurve,
    or a ``{band: LightCurve or (t, y[, dy])}`` mapping, gives a
    MultiBandLightCurve (api.py:47-106)."""
    if isinstance(data, MultiBandLightCurve):
        if domain is None:
            return data
        return MultiBandLightCurve({k: to_input(lc, domain=domain) for k, lc in data.bands.items()},
                                   data.meta)
    if isinstance(data, Mapping):
        return MultiBandLightCurve.from_light_curves(
            {str(k): to_input(v, domain=domain) for k, v in data.items()})
    if isinstance(data, LightCurve):
        return data if domain is None else LightCurve(data.time, data.value, data.error,
                                                      Domain(domain), data.meta)
    if isinstance(data, (tuple, list)) and len(data) in (2, 3):
        t, y = data[0], data[1]
        dy = data[2] if len(data) == 3 else None
        return LightCurve.from_arrays(np.asarray(t), np.asarray(y),
                                      None if dy is None else np.asarray(dy),
                                      domain=Domain(domain) if domain else Domain.MAGNITUDE)
    raise TypeError("expected a LightCurve or a (t, y[, dy]) tuple")


def _settings(settings: Any) -> BLSSettings:
    if settings is None:
        return BLSSettings()
    if isinstance(settings, BLSSettings):
        return settings
    if isinstance(settings, Mapping):
        if "BLS" in settings or "bls" in settings:
            inner = settings.get("BLS", settings.get("bls"))
            return _settings(inner)
        return BLSSettings(**settings)
    raise TypeError(f"settings must be BLSSettings or a mapping, got {type(settings).__name__}")


def periodogram(data: Any, method: str = "BLS", *, backend: str | None = "auto",
                grid: GridSpec | None = None, settings: Any = None,
                domain: Domain | str | None = None, engine=None) -> Periodogram:
    """The BLS periodogram of one light curve (api.py:204-307): flux domain
    (magnitudes converted), the default grid unless ``grid`` is given, peak
    defaults from the settings."""
    m = get_method(method)
    lc = to_input(data, domain=domain)
    s = _settings(settings)
    m.resolve_backend(backend if backend not in (None, "auto") else s.backend)
    if isinstance(lc, MultiBandLightCurve):
        from .multiband import multiband_default_grid
        g = grid or multiband_default_grid(m, lc, s)
        return m.multiband_power(g, lc, s, engine=engine).with_peak_defaults(s)
    single = lc.in_domain(m.natural_domain)
    g = grid or m.default_grid(single, s)
    pg = m.power(g, single, s, engine=engine)
    return pg.with_peak_defaults(s)


__all__ = ["periodogram", "to_input"]

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


def _looks_like_arrays(data: Any) -> bool:
    return isinstance(data, (tuple, list)) and len(data) in (2, 3) and all(
        np.ndim(x) == 1 for x in data)


def _check_bands(bands: Mapping[str, Any], domain: Domain | None) -> None:
    """Every band a LightCurve, all in one domain unless ``domain`` converts them
    (api.py:134-158)."""
    for name, lc in bands.items():
        if not isinstance(lc, LightCurve):
            raise TypeError(f"band {name!r} is a {type(lc).__name__}, not a LightCurve")
    if domain is None and len({lc.domain for lc in bands.values()}) > 1:
        raise ValueError("bands are in different brightness domains; pass domain='magnitude' "
                         "or domain='flux' to convert them all")


def to_input(data: Any, *, columns: Any = None,
             domain: Domain | str | None = None) -> LightCurve | MultiBandLightCurve:
    """A LightCurve or MultiBandLightCurve from a user input (api.py:47-131): a
    LightCurve/MultiBandLightCurve (converted when ``domain`` is given), a
    ``(t, y[, dy])`` tuple (magnitudes unless ``domain`` says otherwise), a
    ``{band: LightCurve}`` mapping, or a pandas/pyarrow/``{column: array}`` table
    read with column detection -- split into bands when ``columns`` names a band
    column."""
    dom = None if domain is None else Domain(domain)
    if isinstance(data, LightCurve):
        return data if dom is None else data.in_domain(dom)
    if isinstance(data, MultiBandLightCurve):
        _check_bands(data.bands, dom)
        if dom is None:
            return data
        return MultiBandLightCurve({k: lc.in_domain(dom) for k, lc in data.bands.items()},
                                   data.meta)
    if _looks_like_arrays(data):
        t, y = data[0], data[1]
        dy = data[2] if len(data) == 3 else None
        return LightCurve.from_arrays(np.asarray(t), np.asarray(y),
                                      None if dy is None else np.asarray(dy),
                                      domain=dom or Domain.MAGNITUDE)
    band_split = columns is not None and getattr(columns, "band", None) is not None
    if isinstance(data, Mapping):
        values = list(data.values())
        if values and all(isinstance(v, LightCurve) for v in values):
            _check_bands(data, dom)
            bands = data if dom is None else {k: lc.in_domain(dom) for k, lc in data.items()}
            return MultiBandLightCurve.from_light_curves({str(k): v for k, v in bands.items()})
    if band_split:
        return MultiBandLightCurve.from_dataframe(data, columns=columns, domain=dom)
    if isinstance(data, Mapping) or hasattr(data, "columns") or hasattr(data, "column_names"):
        return LightCurve.from_dataframe(data, columns=columns, domain=dom)
    raise TypeError("expected a LightCurve, a MultiBandLightCurve, a (t, y[, dy]) tuple, a "
                    "{band: LightCurve} mapping or a table")


def _settings(settings: Any, cls: type = BLSSettings) -> Any:
    """A settings object of the method's class: None gives the defaults, a mapping
    is read directly or under the method's name (``{"TLS": {...}}``)."""
    if settings is None:
        return cls()
    if isinstance(settings, cls):
        return settings
    if isinstance(settings, Mapping):
        name = cls.__name__[:-len("Settings")]
        for key in (name, name.lower()):
            if key in settings:
                return _settings(settings[key], cls)
        return cls(**settings)
    raise TypeError(f"settings must be {cls.__name__} or a mapping, "
                    f"got {type(settings).__name__}")


def periodogram(data: Any, method: str = "BLS", *, backend: str | None = "auto",
                grid: GridSpec | None = None, settings: Any = None, columns: Any = None,
                domain: Domain | str | None = None, engine=None) -> Periodogram:
    """The BLS or TLS periodogram of one light curve (api.py:204-307): flux domain
    (magnitudes converted), the default grid unless ``grid`` is given, peak
    defaults from the settings."""
    m = get_method(method)
    lc = to_input(data, columns=columns, domain=domain)
    s = _settings(settings, m.settings_cls)
    m.resolve_backend(backend if backend not in (None, "auto") else s.backend)
    if isinstance(lc, MultiBandLightCurve):
        if not m.supports_multiband:
            raise ValueError(f"{m.name} does not support multi-band input")
        from .multiband import multiband_default_grid
        g = grid or multiband_default_grid(m, lc, s)
        return m.multiband_power(g, lc, s, engine=engine).with_peak_defaults(s)
    single = lc.in_domain(m.natural_domain)
    g = grid or m.default_grid(single, s)
    pg = m.power(g, single, s, engine=engine)
    return pg.with_peak_defaults(s)


__all__ = ["periodogram", "to_input"]
